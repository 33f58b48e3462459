/*
 * hqt_step_mex.c -- MATLAB MEX gateway of the B200 RK4 step (include/hqt.h).
 *
 *   [Z1,Z2,Z3,Z4,rhoi,info] = hqt_step_mex(Z1,Z2,Z3,Z4,rhoi,P,nsteps)
 *
 * Replaces the loop body of scripts/simulation/tevol_driven_cluster.m:120-142
 * (and of scripts/simulation/tevol_lattice.m:151-173 with
 * P.remove_winding = 0) for `nsteps` steps.  Z1..Z4 and rhoi are the
 * script's workspace arrays, double [nx,ny,nz] (Z1 complex; a real Z1 is
 * promoted), exactly the checkpoint layout of docs/DATA_DICTIONARY.md:27-39.
 * P is a struct with the script constants: L0, L (box lengths, :23-24), mu
 * (:79), vy (boundary A_y = -vy, :86,133), h (:110), remove_winding (1 for
 * the driven script, 0 for the lattice script) and optionally precision
 * (0 FP64, 1 mixed) and filter (default 1).
 *
 * Inputs are not modified (MATLAB arrays are copy-on-write): the outputs are
 * fresh arrays.  info = [steps_done, last_winding].  A non-finite step raises
 * hqt:NonfiniteEvolution, the identifier the reference's smoke test gives
 * the NaN exit of tevol_driven_cluster.m:182-185.
 *
 * Build (interleaved complex API):
 *   mex -R2018a hqt_step_mex.c -I<repo>/include -L<pkg dir> -lhqt
 */
#include <stdint.h>
#include <string.h>

#include "mex.h"
#include "hqt.h"

static hqt_ctx *g_ctx = NULL;
static hqt_params g_cur;

static void release(void) {
    hqt_destroy(g_ctx);
    g_ctx = NULL;
}

static double field_or(const mxArray *P, const char *name, int required, double dflt) {
    const mxArray *f = mxGetField(P, 0, name);
    if (!f) {
        if (required) mexErrMsgIdAndTxt("hqt:BadParams", "P has no field %s", name);
        return dflt;
    }
    return mxGetScalar(f);
}

static void check_field(const mxArray *a, int idx, const mwSize *dims) {
    if (!mxIsDouble(a)) mexErrMsgIdAndTxt("hqt:Args", "input %d must be double", idx + 1);
    if (mxGetNumberOfDimensions(a) != 3)
        mexErrMsgIdAndTxt("hqt:Args", "input %d must be [nx,ny,nz]", idx + 1);
    const mwSize *d = mxGetDimensions(a);
    if (d[0] != dims[0] || d[1] != dims[1] || d[2] != dims[2])
        mexErrMsgIdAndTxt("hqt:Args", "input %d does not match the size of Z1", idx + 1);
    if (idx > 0 && mxIsComplex(a)) mexErrMsgIdAndTxt("hqt:Args", "input %d must be real", idx + 1);
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    if (nrhs != 7) mexErrMsgIdAndTxt("hqt:Args", "7 inputs expected");
    if (nlhs > 6) mexErrMsgIdAndTxt("hqt:Args", "at most 6 outputs");
    if (!mxIsStruct(prhs[5])) mexErrMsgIdAndTxt("hqt:Args", "input 6 must be a struct");
    if (mxGetNumberOfDimensions(prhs[0]) != 3)
        mexErrMsgIdAndTxt("hqt:Args", "Z1 must be [nx,ny,nz]");
    const mwSize *dims = mxGetDimensions(prhs[0]);
    for (int i = 0; i < 5; ++i) check_field(prhs[i], i, dims);
    const double ns = mxGetScalar(prhs[6]);
    if (!(ns >= 0)) mexErrMsgIdAndTxt("hqt:Args", "nsteps must be >= 0");

    hqt_params p;
    memset(&p, 0, sizeof(p));
    p.nx = (int32_t)dims[0];
    p.ny = (int32_t)dims[1];
    p.nz = (int32_t)dims[2];
    p.Lx = field_or(prhs[5], "L0", 1, 0.0);
    p.Ly = field_or(prhs[5], "L", 1, 0.0);
    p.mu = field_or(prhs[5], "mu", 1, 0.0);
    p.vy = field_or(prhs[5], "vy", 1, 0.0);
    p.dt = field_or(prhs[5], "h", 1, 0.0);
    p.remove_winding = (int32_t)field_or(prhs[5], "remove_winding", 1, 1.0);
    p.precision = (int32_t)field_or(prhs[5], "precision", 0, HQT_FP64);
    p.apply_filter = (int32_t)field_or(prhs[5], "filter", 0, 1.0);
    if (!g_ctx || memcmp(&p, &g_cur, sizeof(p)) != 0) { /* one context per set-up */
        release();
        if (hqt_create(&p, 0, &g_ctx) != HQT_OK)
            mexErrMsgIdAndTxt("hqt:Create", "%s", hqt_last_error(NULL));
        g_cur = p;
        mexAtExit(release);
    }
    for (int i = 0; i < 5; ++i) plhs[i] = mxDuplicateArray(prhs[i]);
    if (!mxIsComplex(plhs[0]) && !mxMakeArrayComplex(plhs[0]))
        mexErrMsgIdAndTxt("hqt:Args", "cannot make Z1 complex");
    hqt_diag info;
    memset(&info, 0, sizeof(info));
    const int rc = hqt_step(g_ctx, (double *)mxGetComplexDoubles(plhs[0]),
                            mxGetDoubles(plhs[1]), mxGetDoubles(plhs[2]),
                            mxGetDoubles(plhs[3]), mxGetDoubles(plhs[4]), (int64_t)ns, &info);
    if (rc == HQT_ENONFINITE)
        mexErrMsgIdAndTxt("hqt:NonfiniteEvolution", "Evolution produced NaNs (step %lld).",
                          (long long)info.nonfinite_step);
    if (rc != HQT_OK) mexErrMsgIdAndTxt("hqt:Step", "%s", hqt_last_error(g_ctx));
    if (nlhs > 5) {
        plhs[5] = mxCreateDoubleMatrix(1, 2, mxREAL);
        double *o = mxGetDoubles(plhs[5]);
        o[0] = (double)info.steps_done;
        o[1] = (double)info.last_winding;
    }
}
