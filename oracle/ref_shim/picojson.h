/*
 * Stand-in for the picojson header (an empty git submodule in the
 * reference) so that include/cfg.hpp parses: Cfg declares a member
 * function returning picojson::value.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef PCG_REF_SHIM_PICOJSON_H
#define PCG_REF_SHIM_PICOJSON_H
namespace picojson {
class value {};
}  // namespace picojson
#endif
