/*
 * Hand-written stand-in for the autoconf-generated `include/defines.hpp` of
 * PiCoPiC (configure.ac:96-122, 226-295).  TEST INFRASTRUCTURE ONLY: it lets
 * oracle/Makefile.ref compile the reference's own hot-path sources where
 * they lie, so that the compiled reference can pin the oracle.
 *
 * Always-on switches mirror the reference defaults (Yee solver, PML on,
 * REL_LIMIT = 5e7 m/s, flat plasma, thermal velocities).  The pusher and
 * the current-deposition switch come from the compiler command line
 * (-DSWITCH_PUSHER_...=true, -DSWITCH_CCS_...=true), one library per pair.
 */
#ifndef PCG_REF_SHIM_DEFINES_HPP
#define PCG_REF_SHIM_DEFINES_HPP

#define SWITCH_MAXWELL_SOLVER_YEE true
#define REL_LIMIT 5e7
#define ENABLE_PML true
#define SWITCH_PLASMA_SPATIAL_FLAT true
#define SWITCH_PLASMA_VELOCITY_THERMAL true
#define ENABLE_SINGLETHREAD true

#if !defined(SWITCH_PUSHER_BORIS) && !defined(SWITCH_PUSHER_BORIS_ADAPTIVE) && \
    !defined(SWITCH_PUSHER_BORIS_RELATIVISTIC) && !defined(SWITCH_PUSHER_VAY) && \
    !defined(SWITCH_PUSHER_HC)
#define SWITCH_PUSHER_BORIS_RELATIVISTIC true
#endif

#if !defined(SWITCH_CCS_VB) && !defined(SWITCH_CCS_ZIGZAG)
#define SWITCH_CCS_VB true
#endif

#define PACKAGE_VERSION "reference-hot-path"
#define CXXFLAGS ""

#endif
