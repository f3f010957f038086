/*
 * Replacement top-level header used ONLY to compile the reference SHAPE CPU
 * sources in place (oracle/_ref build; test infrastructure, never shipped).
 *
 * The reference's own src/shape/head.h cannot be used here:
 *   - it includes cfitsio through an absolute path of the original author's
 *     machine (src/shape/head.h:29) and cfitsio is not installed;
 *   - it includes ../HybridCode/hybrid.h (src/shape/head.h:36), a directory
 *     that is missing from the reference tree;
 *   - it includes the CUDA-C headers of the superseded GPU port
 *     (src/CudaCode/shape-cuda.h etc.), which use __host__/int4/dim3 and do
 *     not compile as plain C.
 * This header pulls in the same plain-C headers from the reference tree (found
 * through -I paths set by oracle/build_ref.sh), a cfitsio stub, and the handful
 * of flags and macros that the C sources take from the GPU headers.
 */
#ifndef SHAPE_REFSHIM_HEAD_H
#define SHAPE_REFSHIM_HEAD_H

#include <stdlib.h>
#include <stdio.h>
#include <math.h>
#include <string.h>
#include <sys/resource.h>
#include <sys/time.h>
#include <sys/types.h>
#include <unistd.h>
#include <pthread.h>
#include <ctype.h>

#include "build.h"
#include "nr.h"
#include "../macros/files.h"
#include "../macros/func.h"
#include "util.h"
#include "astro.h"
#include "pgm.h"
#include "shape2.h"
#include "fitsio.h"
#include "const.h"
#include "hmt.h"

/* Flags and globals that the C sources read (declared in the CUDA header of
 * the GPU port, src/CudaCode/shape-cuda.h:28-49; defined in refstubs.c). */
extern int CUDA, GPU0, GPU1, TIMING, MGPU, PIN, EXP, MFS, HYB;
extern int maxThreadsPerBlock;
extern double *fparstep, *fpartol, *fparabstol, **fpntr;
extern int *fpartype;

/* Allocation macros of the GPU header, mapped to host allocation. */
#define gpuErrchk(ans) (ans)
#define cudaCalloc(A, B, C) do { *(A) = calloc((B), (C)); } while (0)
#define cudaCalloc1(A, B, C) do { *(A) = calloc((B), (C)); } while (0)

#endif
