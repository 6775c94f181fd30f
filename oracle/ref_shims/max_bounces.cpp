// Oracle build shim: storage of the runtime bounce cap declared in max_bounces.h.
#include "max_bounces.h"

extern "C" unsigned int ph_oracle_max_ray_bounces = 10000;
