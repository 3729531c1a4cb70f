/* libipcb200_direct: sparse Cholesky solve of the 3x3-block Newton system.
 *
 * Replaces the reference's direct path, time_integrator_base.py:470-500
 * (``solve_ldlt``: BSR -> scalar CSR by ``bsr_to_scalar_csr``
 * (time_integrator_base.py:33-62), then ``DirectSolverDevice``
 * ``analyze_pattern`` / ``factorize`` / ``solve`` from dxslv/cuDSS), with the
 * same three phases on cuSOLVER's device Cholesky (csrchol), which is present
 * in this CUDA toolkit while cuDSS is not.  A fill-reducing ordering is
 * computed on the block graph (so each 3x3 block stays together) and the
 * permuted scalar CSR is gathered from the BSR values on the device.
 *
 * Kept in its own library so that libipcb200 does not depend on cuSOLVER.
 * Pointers are device pointers unless stated otherwise; the BSR arrays are
 * the canonical ones of ipcb_bsr_from_triplets (sorted, symmetric pattern).
 * Return 0 on success, IPCB_E_ARG / IPCB_E_CUDA (include/ipcb.h) or
 * IPCB_E_SINGULAR when the factorisation meets a zero/negative pivot. */
#ifndef IPCB_DIRECT_H
#define IPCB_DIRECT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IPCB_E_SINGULAR 3

/* orderings of the block graph */
#define IPCB_ORDER_NONE 0
#define IPCB_ORDER_SYMRCM 1
#define IPCB_ORDER_SYMAMD 2
#define IPCB_ORDER_METIS 3

typedef void* ipcb_direct_handle;
typedef void* ipcb_direct_stream;

const char* ipcb_direct_last_error(void);
int ipcb_direct_create(ipcb_direct_handle* out);
int ipcb_direct_destroy(ipcb_direct_handle h);
/* Symbolic phase (DirectSolverDevice.analyze_pattern): n_blocks block rows,
 * offsets int32[n_blocks + 1], columns int32[nnz_blocks].  fp64 selects the
 * factor type (0: float, 1: double).  Synchronises the stream (the ordering
 * runs on the host). */
int ipcb_direct_analyze(ipcb_direct_handle h, int n_blocks, int nnz_blocks, const int* offsets, const int* columns,
                        int fp64, int ordering, ipcb_direct_stream s);
/* Numeric phase (factorize): values scalar[9 * nnz_blocks] of the analysed
 * pattern, in the factor type.  Synchronises to read the pivot check. */
int ipcb_direct_factor(ipcb_direct_handle h, const void* values, ipcb_direct_stream s);
/* x = A^-1 b for b, x scalar[3 * n_blocks] (solve). */
int ipcb_direct_solve(ipcb_direct_handle h, const void* b, void* x, ipcb_direct_stream s);
/* Bytes of the factor's internal data (fill) and of the work buffer, after
 * analyze; host pointers, either may be NULL. */
int ipcb_direct_sizes(ipcb_direct_handle h, size_t* factor_bytes, size_t* work_bytes);

#ifdef __cplusplus
}
#endif
#endif
