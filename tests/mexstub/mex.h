/* Declarations-only stand-in for MATLAB's mex.h (R2018a interleaved-complex API), enough for a
 * syntax and type check of the MEX gateway; MATLAB's own header is used for the real build. */
#pragma once
#include <stddef.h>
#include <stdint.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxUNKNOWN_CLASS, mxLOGICAL_CLASS, mxDOUBLE_CLASS, mxSINGLE_CLASS, mxUINT8_CLASS, mxUINT16_CLASS,
               mxUINT32_CLASS } mxClassID;
typedef enum { mxREAL, mxCOMPLEX } mxComplexity;
typedef struct { double real, imag; } mxComplexDouble;
typedef struct { float real, imag; } mxComplexSingle;
extern "C" {
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID c, mxComplexity flag);
mxArray* mxCreateLogicalArray(mwSize ndim, const mwSize* dims);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag);
mxArray* mxCreateDoubleScalar(double v);
void mxDestroyArray(mxArray* a);
mxClassID mxGetClassID(const mxArray* a);
mxComplexDouble* mxGetComplexDoubles(const mxArray* a);
mxComplexSingle* mxGetComplexSingles(const mxArray* a);
void* mxGetData(const mxArray* a);
double* mxGetPr(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
size_t mxGetElementSize(const mxArray* a);
mxArray* mxGetField(const mxArray* a, size_t i, const char* name);
double mxGetScalar(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize n);
bool mxIsChar(const mxArray* a);
bool mxIsEmpty(const mxArray* a);
bool mxIsStruct(const mxArray* a);
}
