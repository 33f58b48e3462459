/* Minimal declarations of the MATLAB MEX C API (R2018a interleaved complex)
 * used by hqt_step_mex.c, so that the gateway can be compile-checked where
 * MATLAB is not installed.  Test infrastructure only: declarations, no
 * implementation. */
#ifndef HQT_TEST_MEX_STUB_H
#define HQT_TEST_MEX_STUB_H
#include <stddef.h>
#include <stdbool.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxREAL, mxCOMPLEX } mxComplexity;
typedef struct { double real, imag; } mxComplexDouble;
typedef double mxDouble;

const mxArray *mxGetField(const mxArray *pa, size_t i, const char *fieldname);
double mxGetScalar(const mxArray *pa);
bool mxIsDouble(const mxArray *pa);
bool mxIsComplex(const mxArray *pa);
bool mxIsStruct(const mxArray *pa);
size_t mxGetNumberOfDimensions(const mxArray *pa);
const mwSize *mxGetDimensions(const mxArray *pa);
mxArray *mxDuplicateArray(const mxArray *in);
int mxMakeArrayComplex(mxArray *pa);
mxComplexDouble *mxGetComplexDoubles(const mxArray *pa);
mxDouble *mxGetDoubles(const mxArray *pa);
mxArray *mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity flag);
void mexErrMsgIdAndTxt(const char *identifier, const char *err_msg, ...);
int mexAtExit(void (*exit_fcn)(void));
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
#endif
