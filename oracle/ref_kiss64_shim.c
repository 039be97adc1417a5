/* Build shim -- TEST INFRASTRUCTURE ONLY: the reference's prj/common/kiss_fft.c
 * compiled with a double scalar, to pair with ref_prj64_shim.c. */
#include <stdlib.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <limits.h>
#include <alloca.h>
#define kiss_fft_scalar double
#include "common/kiss_fft.c"
