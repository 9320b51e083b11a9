/*
 * Force-included when the reference projector sources are compiled by
 * oracle/Makefile.  It replaces the reference's spdlog wrapper
 * (hrrt_common/my_spdlog.hpp:44-67) with no-op logging and maps LOG_EXIT to
 * exit(1), which is what the wrapper does after logging.  Nothing here changes
 * arithmetic.  This file is test infrastructure: it is compiled only into
 * oracle/_ref/libhrrt_ref.so, never into the product library.
 */
#pragma once
#include <stdio.h>
#include <stdlib.h>
#include <alloca.h>

#define LOG_INFO(...)  ((void)0)
#define LOG_ERROR(...) ((void)0)
#define LOG_DEBUG(...) ((void)0)
#define LOG_TRACE(...) ((void)0)
#define LOG_EXIT(...)  exit(1)
