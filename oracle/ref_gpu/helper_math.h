// Stand-in for the CUDA samples' helper_math.h, which the reference's
// particle_hash_kernel.cu includes; the kernels it is built for here use only
// the vector constructors of the toolkit.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <vector_functions.h>
