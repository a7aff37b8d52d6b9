// qdldl.h -- the QDLDL API (types and the three calls the reference makes,
// qdldl_helper.cuh:62-180) bound to the oracle's own implementation in
// oracle/ldl.c (written from Davis's up-looking elimination-tree LDL^T,
// ACM TOMS 31(4), 2005).  The qdldl submodule is empty in the reference tree
// (.gitmodules:7-9); the reference builds it with FP32 values and int32
// indices (README.md:14-19).  Test infrastructure only.
#pragma once
#include <stdint.h>

typedef int32_t QDLDL_int;
typedef float QDLDL_float;
typedef unsigned char QDLDL_bool;

#ifdef __cplusplus
extern "C" {
#endif
QDLDL_int QDLDL_etree(const QDLDL_int n, const QDLDL_int *Ap, const QDLDL_int *Ai, QDLDL_int *work, QDLDL_int *Lnz,
                      QDLDL_int *etree);
QDLDL_int QDLDL_factor(const QDLDL_int n, const QDLDL_int *Ap, const QDLDL_int *Ai, const QDLDL_float *Ax,
                       QDLDL_int *Lp, QDLDL_int *Li, QDLDL_float *Lx, QDLDL_float *D, QDLDL_float *Dinv,
                       const QDLDL_int *Lnz, const QDLDL_int *etree, QDLDL_bool *bwork, QDLDL_int *iwork,
                       QDLDL_float *fwork);
void QDLDL_solve(const QDLDL_int n, const QDLDL_int *Lp, const QDLDL_int *Li, const QDLDL_float *Lx,
                 const QDLDL_float *Dinv, QDLDL_float *x);
#ifdef __cplusplus
}
#endif
