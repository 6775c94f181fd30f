// Oracle build shim (test infrastructure only, never linked into the product).
//
// The reference fixes the bounce cap at compile time (`#define MAX_RAY_BOUNCES 10000`,
// Engine/Source/Core/Estimator/BNEEPTEstimator.cpp:27 and BVPTEstimator.cpp:19). The oracle build
// compiles a generated copy of those two TUs (made at build time by oracle/Makefile.ref, never
// committed) in which that one line reads the cap from this runtime variable instead, so a
// single oracle library renders both the uncapped reference behaviour (default 10000) and the
// depth-capped benchmark workloads. No other line of the estimators is changed.
#pragma once

extern "C" unsigned int ph_oracle_max_ray_bounces;
