/*
 * Build shim for the FP64 variant of the reference projector -- TEST
 * INFRASTRUCTURE ONLY.  It compiles the reference's unchanged prj/cpuPrj.c
 * (found on the include path) with its scalar type widened to double:
 * prj/prj.h:36-40 hard-codes `typedef float ft`, so every `float` spelled in
 * the reference sources is redefined after the system headers have been read.
 * Float literals such as the pi constant (prj/prj.h:9) keep their type, as in
 * the reference's own double build.
 */
#include <stdlib.h>
#include <math.h>
#include <stdio.h>
#include <time.h>
#include <limits.h>
#include <stddef.h>
#include <string.h>
#include <float.h>
#include <pthread.h>
#include <alloca.h>
#define kiss_fft_scalar double
#define float double
#include "cpuPrj.c"
