/*
 * Build configuration used when the upstream PDP3 sources are compiled as the
 * test oracle (oracle/_ref).  The upstream project generates this header with
 * autoconf; autoconf is not available here, so the few macros the hot-path
 * sources read are set by hand.  The pusher macro (PUSHER_BORIS_RELATIVISTIC,
 * PUSHER_BORIS_ADAPTIVE or PUSHER_VAY) and TESTMODE are passed with -D by
 * oracle/Makefile so one header serves every oracle variant.
 *
 * IEEE build: no -ffast-math and no -mavx, so lib::sq_rt is plain sqrt()
 * (src/lib.cpp:27-35 switches to an AVX path only when __AVX__ is defined).
 */
#pragma once

#ifndef REL_LIMIT
#define REL_LIMIT 5e7
#endif

#define TEMPERATURE_POSTPROC_NONE true
#define PACKAGE_NAME "pdp3"
#define PACKAGE_STRING "pdp3 (oracle build)"
#define PACKAGE_VERSION "oracle"
