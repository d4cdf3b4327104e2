/* LINK-CHECK STUB -- not MATLAB's header, and nothing here is ever run.
 *
 * Declares the part of MATLAB's documented C matrix API (mxArray access and
 * allocation) that the reference's MEX gateway (src/speigs_mex.c) calls, so
 * the gateway can be compiled and linked against this project's
 * libspeigs.so without MATLAB.  The symbols stay undefined in the linked
 * object; a MATLAB installation provides them at load time.  Types follow
 * the documented 64-bit (-largeArrayDims) API.
 */
#ifndef SPEIGS_MEXSTUB_MATRIX_H
#define SPEIGS_MEXSTUB_MATRIX_H
#include <stddef.h>
#include <stdbool.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef struct { double real, imag; } mxComplexDouble;

bool    mxIsSparse(const mxArray *a);
bool    mxIsDouble(const mxArray *a);
bool    mxIsComplex(const mxArray *a);
bool    mxIsChar(const mxArray *a);
bool    mxIsStruct(const mxArray *a);
bool    mxIsEmpty(const mxArray *a);
bool    mxIsNumeric(const mxArray *a);
size_t  mxGetM(const mxArray *a);
size_t  mxGetN(const mxArray *a);
mwIndex *mxGetJc(const mxArray *a);
mwIndex *mxGetIr(const mxArray *a);
double  *mxGetPr(const mxArray *a);
double  *mxGetPi(const mxArray *a);
double  *mxGetDoubles(const mxArray *a);
mxComplexDouble *mxGetComplexDoubles(const mxArray *a);
double  mxGetScalar(const mxArray *a);
int     mxGetString(const mxArray *a, char *buf, mwSize len);
mxArray *mxGetField(const mxArray *a, mwIndex i, const char *name);
void    mxSetField(mxArray *a, mwIndex i, const char *name, mxArray *value);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray *mxCreateDoubleScalar(double v);
mxArray *mxCreateString(const char *s);
mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **names);
void    mxDestroyArray(mxArray *a);
void   *mxMalloc(mwSize bytes);
void   *mxCalloc(mwSize n, mwSize size);
void    mxFree(void *p);
#endif
