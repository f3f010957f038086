/*
 * Definitions that the reference SHAPE CPU sources need at link time but that
 * live outside the files compiled into oracle/_ref (test infrastructure only).
 *
 *  - mode flags defined next to main() in src/shape/shape-cuda-v1.0.c:12-23
 *    (main itself is not linked: the harness calls the hot-path functions);
 *  - cfitsio entry points used only by the FITS frame reader
 *    (src/shape/read_dat.c), which the harness never reaches;
 *  - cudaSetDevice, referenced by the pthread helpers of src/shape/read_mod.c.
 * Each stub reports failure; none is on the evaluated path.
 */
#include <stdio.h>
#include <stdlib.h>

int CUDA = 0, TIMING = 0, GPU0 = 0, GPU1 = 0, MGPU = 0, PIN = 0;
int maxThreadsPerBlock = 0, HMT = 0, HMT_threads = 1, EXP = 0, MFS = 0, HYB = 0;

typedef struct { int unused; } fitsfile;

static int refstub_fail(const char *name)
{
    fprintf(stderr, "oracle/_ref: %s is not available in this build\n", name);
    return 1;
}

int fits_open_file(fitsfile **f, const char *n, int m, int *s) { (void)f; (void)n; (void)m; *s = 1; return refstub_fail("fits_open_file"); }
int fits_close_file(fitsfile *f, int *s) { (void)f; *s = 1; return refstub_fail("fits_close_file"); }
int fits_read_key_lng(fitsfile *f, const char *k, long *v, char *c, int *s) { (void)f; (void)k; (void)v; (void)c; *s = 1; return refstub_fail("fits_read_key_lng"); }
int fits_read_keys_lng(fitsfile *f, const char *k, int a, int b, long *v, int *nf, int *s) { (void)f; (void)k; (void)a; (void)b; (void)v; (void)nf; *s = 1; return refstub_fail("fits_read_keys_lng"); }
int fits_read_img(fitsfile *f, int t, long a, long n, void *nv, void *arr, int *an, int *s) { (void)f; (void)t; (void)a; (void)n; (void)nv; (void)arr; (void)an; *s = 1; return refstub_fail("fits_read_img"); }
void fits_report_error(FILE *st, int s) { (void)st; (void)s; refstub_fail("fits_report_error"); }
int cudaSetDevice(int d) { (void)d; return refstub_fail("cudaSetDevice"); }
