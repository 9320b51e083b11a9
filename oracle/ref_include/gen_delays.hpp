/*
 * Stands in for gen_delays.hpp, which gen_delays_lib/gen_delays_lib.cpp:40
 * includes and the reference tree does not contain.  It declares only the
 * four file names gen_delays_lib.cpp reads (their definitions are commented
 * out there, :56-59); oracle/lmhist_ref_main.cpp defines them empty.  Test
 * infrastructure only.
 */
#pragma once
#include <boost/filesystem.hpp>

extern boost::filesystem::path g_coincidence_histogram_file;
extern boost::filesystem::path g_crystal_singles_file;
extern boost::filesystem::path g_delayed_coincidence_file;
extern boost::filesystem::path g_output_csings_file;
