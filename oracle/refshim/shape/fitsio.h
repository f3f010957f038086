/*
 * Minimal cfitsio stand-in used ONLY to compile the reference SHAPE CPU
 * sources (oracle/_ref build). cfitsio is not installed in this image; the
 * reference uses it only in the FITS delay-Doppler frame reader
 * (src/shape/read_dat.c), which is off the model-evaluation path. Every
 * function here reports failure.
 */
#ifndef SHAPE_REFSHIM_FITSIO_H
#define SHAPE_REFSHIM_FITSIO_H

typedef struct { int unused; } fitsfile;

#define READONLY 0
#define READWRITE 1
#define TBYTE 11
#define TSHORT 21
#define TINT 31
#define TLONG 41
#define TFLOAT 42
#define TDOUBLE 82
#define FLEN_ERRMSG 81

int fits_open_file(fitsfile **fptr, const char *name, int mode, int *status);
int fits_close_file(fitsfile *fptr, int *status);
int fits_read_key_lng(fitsfile *fptr, const char *key, long *val, char *comm, int *status);
int fits_read_keys_lng(fitsfile *fptr, const char *key, int n0, int n, long *vals, int *nfound, int *status);
int fits_read_img(fitsfile *fptr, int type, long first, long n, void *nulv, void *arr, int *anynul, int *status);
void fits_report_error(FILE *stream, int status);

#endif
