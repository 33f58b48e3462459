/* A tiny stand-in for the MATLAB MEX runtime (test infrastructure only): the
 * mx* functions hqt_step_mex.c uses, over plain heap arrays, and a main() that
 * plays MATLAB's part of
 *
 *   [Z1,Z2,Z3,Z4,rhoi,info] = hqt_step_mex(Z1,Z2,Z3,Z4,rhoi,P,nsteps)
 *
 * Usage: fake_mex <in.bin> <out.bin> nx ny nz L0 L mu vy h remove_winding nsteps
 * in.bin holds Z1 (interleaved complex), Z2, Z3, Z4, rhoi as column-major
 * doubles; out.bin receives the five outputs in the same layout followed by
 * info (2 doubles).  A mexErrMsgIdAndTxt prints its identifier and exits 3. */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
    int is_struct;
    size_t ndim;
    mwSize dims[3];
    int complex_;
    double *re;             /* real data, or interleaved complex when complex_ */
    int nfields;
    const char *names[16];
    mxArray *values[16];
};

static size_t numel(const mxArray *a) {
    size_t n = 1;
    for (size_t i = 0; i < a->ndim; ++i) n *= a->dims[i];
    return n;
}

static mxArray *new_double(size_t ndim, const mwSize *dims, int cplx) {
    mxArray *a = calloc(1, sizeof(mxArray));
    a->ndim = ndim;
    for (size_t i = 0; i < ndim; ++i) a->dims[i] = dims[i];
    a->complex_ = cplx;
    a->re = calloc(numel(a) * (cplx ? 2 : 1), sizeof(double));
    return a;
}

static mxArray *scalar(double v) {
    mwSize d[2] = {1, 1};
    mxArray *a = new_double(2, d, 0);
    a->re[0] = v;
    return a;
}

const mxArray *mxGetField(const mxArray *pa, size_t i, const char *name) {
    (void)i;
    for (int k = 0; k < pa->nfields; ++k)
        if (strcmp(pa->names[k], name) == 0) return pa->values[k];
    return NULL;
}
double mxGetScalar(const mxArray *pa) { return pa->re[0]; }
bool mxIsDouble(const mxArray *pa) { return !pa->is_struct; }
bool mxIsComplex(const mxArray *pa) { return pa->complex_ != 0; }
bool mxIsStruct(const mxArray *pa) { return pa->is_struct != 0; }
size_t mxGetNumberOfDimensions(const mxArray *pa) { return pa->ndim; }
const mwSize *mxGetDimensions(const mxArray *pa) { return pa->dims; }
mxArray *mxDuplicateArray(const mxArray *in) {
    mxArray *a = new_double(in->ndim, in->dims, in->complex_);
    memcpy(a->re, in->re, numel(in) * (in->complex_ ? 2 : 1) * sizeof(double));
    return a;
}
int mxMakeArrayComplex(mxArray *pa) {
    const size_t n = numel(pa);
    double *z = calloc(2 * n, sizeof(double));
    for (size_t i = 0; i < n; ++i) z[2 * i] = pa->re[i];
    free(pa->re);
    pa->re = z;
    pa->complex_ = 1;
    return 1;
}
mxComplexDouble *mxGetComplexDoubles(const mxArray *pa) {
    return pa->complex_ ? (mxComplexDouble *)pa->re : NULL;
}
mxDouble *mxGetDoubles(const mxArray *pa) { return pa->complex_ ? NULL : pa->re; }
mxArray *mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity flag) {
    mwSize d[2] = {m, n};
    return new_double(2, d, flag == mxCOMPLEX);
}
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
    va_list ap;
    fprintf(stderr, "%s: ", id);
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fprintf(stderr, "\n");
    exit(3);
}
static void (*g_atexit)(void) = NULL;
int mexAtExit(void (*f)(void)) {
    g_atexit = f;
    return 0;
}

int main(int argc, char **argv) {
    if (argc != 13) {
        fprintf(stderr, "usage: fake_mex in out nx ny nz L0 L mu vy h rw nsteps\n");
        return 1;
    }
    mwSize d[3] = {(mwSize)atol(argv[3]), (mwSize)atol(argv[4]), (mwSize)atol(argv[5])};
    mxArray *in[7];
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 1;
    for (int i = 0; i < 5; ++i) {
        in[i] = new_double(3, d, i == 0);
        const size_t n = numel(in[i]) * (i == 0 ? 2 : 1);
        if (fread(in[i]->re, sizeof(double), n, f) != n) return 1;
    }
    fclose(f);
    mxArray *P = calloc(1, sizeof(mxArray));
    P->is_struct = 1;
    const char *names[] = {"L0", "L", "mu", "vy", "h", "remove_winding"};
    for (int k = 0; k < 6; ++k) {
        P->names[k] = names[k];
        P->values[k] = scalar(atof(argv[6 + k]));
    }
    P->nfields = 6;
    in[5] = P;
    in[6] = scalar(atof(argv[12]));
    mxArray *out[6] = {0};
    mexFunction(6, out, 7, (const mxArray **)in);
    f = fopen(argv[2], "wb");
    if (!f) return 1;
    for (int i = 0; i < 6; ++i)
        fwrite(out[i]->re, sizeof(double), numel(out[i]) * (out[i]->complex_ ? 2 : 1), f);
    fclose(f);
    /* the inputs must be untouched (copy-on-write) */
    if (g_atexit) g_atexit();
    return 0;
}
