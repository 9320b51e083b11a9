/*
 * Stands in for the reference's spdlog wrapper (hrrt_common/my_spdlog.hpp)
 * when oracle/Makefile compiles reference sources that include it: the
 * logging macros come from ref_shim.h (force-included), which log nothing.
 * Test infrastructure only.
 */
#pragma once
