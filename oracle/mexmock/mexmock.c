/* mexmock.c -- TEST INFRASTRUCTURE ONLY: the minimal MEX API of mex.h. */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
    mxClassID cls;
    size_t m, n;
    void *data;
    int nfields;
    char **names;
    mxArray **values;
};

static int g_errors = 0;

static mxArray *alloc_array(mxClassID cls, size_t m, size_t n, size_t elem)
{
    mxArray *a = (mxArray *)calloc(1, sizeof *a);
    a->cls = cls;
    a->m = m;
    a->n = n;
    a->data = calloc(m * n ? m * n : 1, elem);
    return a;
}

mxArray *mxCreateNumericMatrix(size_t m, size_t n, mxClassID cls, mxComplexity cx)
{
    (void)cx;
    return alloc_array(cls, m, n, cls == mxSINGLE_CLASS ? sizeof(float) : sizeof(double));
}

mxArray *mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity cx)
{
    return mxCreateNumericMatrix(m, n, mxDOUBLE_CLASS, cx);
}

double *mxGetPr(const mxArray *a) { return (double *)a->data; }
void *mxGetData(const mxArray *a) { return a->data; }
int mxIsDouble(const mxArray *a) { return a && a->cls == mxDOUBLE_CLASS; }
int mxIsSingle(const mxArray *a) { return a && a->cls == mxSINGLE_CLASS; }

char *mxArrayToString(const mxArray *a)
{
    if (!a || a->cls != mxCHAR_CLASS) return NULL;
    size_t len = a->m * a->n;
    char *s = (char *)malloc(len + 1);
    memcpy(s, a->data, len);
    s[len] = 0;
    return s;
}

mxArray *mxGetField(const mxArray *a, size_t index, const char *name)
{
    if (!a || a->cls != mxSTRUCT_CLASS || index != 0) return NULL;
    for (int i = 0; i < a->nfields; i++)
        if (!strcmp(a->names[i], name)) return a->values[i];
    return NULL;
}

double mxGetScalar(const mxArray *a)
{
    if (!a || a->m * a->n == 0) return 0.0;
    if (a->cls == mxSINGLE_CLASS) return ((float *)a->data)[0];
    return ((double *)a->data)[0];
}

size_t mxGetNumberOfElements(const mxArray *a) { return a ? a->m * a->n : 0; }
void mxFree(void *p) { free(p); }

int mexPrintf(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    int r = vprintf(fmt, ap);
    va_end(ap);
    fflush(stdout);
    return r;
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...)
{
    (void)id;
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    g_errors++;
}

mxArray *mock_numeric(size_t m, size_t n, int single, const void *data)
{
    mxArray *a = mxCreateNumericMatrix(m, n, single ? mxSINGLE_CLASS : mxDOUBLE_CLASS, mxREAL);
    if (data) memcpy(a->data, data, m * n * (single ? sizeof(float) : sizeof(double)));
    return a;
}

mxArray *mock_string(const char *s)
{
    size_t len = strlen(s);
    mxArray *a = alloc_array(mxCHAR_CLASS, 1, len, 1);
    memcpy(a->data, s, len);
    return a;
}

mxArray *mock_struct(int nfields, const char **names, mxArray **values)
{
    mxArray *a = (mxArray *)calloc(1, sizeof *a);
    a->cls = mxSTRUCT_CLASS;
    a->m = a->n = 1;
    a->nfields = nfields;
    a->names = (char **)calloc(nfields, sizeof(char *));
    a->values = (mxArray **)calloc(nfields, sizeof(mxArray *));
    for (int i = 0; i < nfields; i++) {
        a->names[i] = strdup(names[i]);
        a->values[i] = values[i];
    }
    return a;
}

void mock_destroy(mxArray *a)
{
    if (!a) return;
    if (a->cls == mxSTRUCT_CLASS) {
        for (int i = 0; i < a->nfields; i++) {
            free(a->names[i]);
            mock_destroy(a->values[i]);
        }
        free(a->names);
        free(a->values);
    }
    free(a->data);
    free(a);
}

int mock_error_count(void) { return g_errors; }
