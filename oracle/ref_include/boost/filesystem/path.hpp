/* See boost/filesystem.hpp beside this file (test infrastructure only). */
#pragma once
#include "../filesystem.hpp"
