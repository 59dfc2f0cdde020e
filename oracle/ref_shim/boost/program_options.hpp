// The one boost::program_options name the reference's configuration.h
// declares (the return type of parse_configs).  TEST INFRASTRUCTURE ONLY:
// configuration.cpp itself is not compiled into the checker; the harness sets
// the global `config` directly.
#ifndef QUEST_REF_SHIM_BOOST_PROGRAM_OPTIONS
#define QUEST_REF_SHIM_BOOST_PROGRAM_OPTIONS
namespace boost {
namespace program_options {
class variables_map {};
}  // namespace program_options
}  // namespace boost
#endif
