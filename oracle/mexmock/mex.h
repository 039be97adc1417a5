/*
 * mex.h -- TEST INFRASTRUCTURE ONLY: a minimal stand-in for MATLAB's MEX API
 * (MATLAB is not installed here), enough to compile and drive the reference's
 * own MEX gateways prj/mPrj.c and prj/mParPrj.c against libctprj.so.  Arrays
 * are column-major like MATLAB's; struct arrays hold one element.
 */
#ifndef MEXMOCK_MEX_H
#define MEXMOCK_MEX_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS, mxSINGLE_CLASS, mxCHAR_CLASS, mxSTRUCT_CLASS } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;
typedef struct mxArray_tag mxArray;

mxArray *mxCreateNumericMatrix(size_t m, size_t n, mxClassID cls, mxComplexity cx);
mxArray *mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity cx);
double *mxGetPr(const mxArray *a);
void *mxGetData(const mxArray *a);
int mxIsDouble(const mxArray *a);
int mxIsSingle(const mxArray *a);
char *mxArrayToString(const mxArray *a);
mxArray *mxGetField(const mxArray *a, size_t index, const char *name);
double mxGetScalar(const mxArray *a);
size_t mxGetNumberOfElements(const mxArray *a);
void mxFree(void *p);
int mexPrintf(const char *fmt, ...);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);

/* test helpers */
mxArray *mock_numeric(size_t m, size_t n, int single, const void *data);
mxArray *mock_string(const char *s);
mxArray *mock_struct(int nfields, const char **names, mxArray **values);
void mock_destroy(mxArray *a);
int mock_error_count(void);

#ifdef __cplusplus
}
#endif
#endif
