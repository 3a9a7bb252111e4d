/*
 * Pre-included ahead of every reference translation unit by
 * oracle/ref/Makefile.ref.  The reference declares a global `float *array`
 * (Main.cu:31) and also says `using namespace std` (Main.cuh:32), which makes
 * unqualified `array` ambiguous with std::array under current libstdc++.  This
 * header includes every system header the reference uses first, so their text
 * is already processed, and only then renames the reference's own identifier.
 * No reference source is copied or edited.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <cstdarg>
#include <iostream>
#include <string>
#include <array>
#include <sys/types.h>
#include <sys/stat.h>
#include <unistd.h>
#include <ctype.h>
#include <cufft.h>
#include <math_constants.h>
#include <cuda_runtime.h>
#include <device_launch_parameters.h>
#include <cooperative_groups.h>
#include <omp.h>
#define array fargo_ref_global_array
