// CPU restatement of the CTBB_ICD reconstruction path ("the oracle port").
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product library links or calls this
// code; tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// it (oracle/_ref/liboracle_port.so) as the checker. Each function cites the
// reference file:line it restates. Its outputs are pinned against the
// reference program itself (oracle/_ref/icd_ref built from the reference
// sources) by tests/test_oracle_pin.py and the fixtures in tests/golden/.
#pragma once

#include <stdint.h>

#include "../include/ctbb_icd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct port_ssm port_ssm;

// Stored system matrix, ray-driven like generate_system_matrix.cpp:80-186 and
// generate_system_matrix_ffs.cpp:104-222 (FFS chosen by geom->Phiffs).
port_ssm* port_ssm_build(const ctbb_geom_c* geom);
uint64_t port_ssm_nnz(const port_ssm* s);
// The entries of selected columns on selected (ascending) views only, same
// arithmetic; counts[c * n_views + v] per (column, view), entries written in
// that order up to `capacity`. Returns the total entry count.
uint64_t port_ssm_subset(const ctbb_geom_c* geom, int n_cols, const int64_t* cols, int n_views,
                         const int32_t* views, uint32_t* counts, int32_t* idx, float* w, uint64_t capacity);
void port_ssm_copy(const port_ssm* s, int64_t* colptr, int32_t* idx, float* w);
void port_ssm_free(port_ssm* s);

// Sequential ICD (icd_iteration.cpp:149-274) with the reference penalties
// (penalties.cpp:39-154). x: FP64 image [nz][ny][nx] (in/out); est: FP64
// sinogram estimate (in/out). dumps: optional n_iter * nvox FP64 images
// written after each iteration (iterationN.rcn, icd_iteration.cpp:265-269).
void port_icd(const ctbb_geom_c* geom, const uint64_t* slice_indices, const float* raw,
              const int64_t* colptr, const int32_t* idx, const float* w, double* x, double* est,
              int n_iter, double* dumps);

// rotate_slices_{fixed2rotating,rotating2fixed} (rotate_slices.cpp:48-154)
// with interp2 (interp.h:41-76). direction: +1 fixed->rotating, -1 back.
void port_rotate(const ctbb_geom_c* geom, const double* tube_angles, const uint64_t* slice_indices,
                 float* vol, int direction);

// FP64 forward projection A x with the in-range test of icd_iteration.cpp:205-207.
void port_forward(const ctbb_geom_c* geom, const uint64_t* slice_indices, const int64_t* colptr,
                  const int32_t* idx, const float* w, const double* x, double* out);

// FP64 cost minimised by the reference update rules:
//   quadratic:        1/2 |y - Ax|^2 + lambda/4 sum_q sum_n w (x_q - x_n)^2
//   edge-preserving:  |y - Ax|^2 + lambda/2 sum_q sum_n w rho(x_q - x_n),
//                     rho(t) = |t| - delta ln(1 + |t|/delta)
// data_term / penalty_term receive the two parts (may be NULL).
double port_cost(const ctbb_geom_c* geom, const uint64_t* slice_indices, const float* raw,
                 const int64_t* colptr, const int32_t* idx, const float* w, const double* x,
                 double* data_term, double* penalty_term);

// The reference's penalised one-voxel update (penalties.cpp:61-154) on given
// inputs: x9[9 i] the voxel, x9[9 i + 1 + l] its neighbour l in the order
// {-nx-1, -nx, -nx+1, -1, +1, nx-1, nx, nx+1} (NaN: outside the volume).
void port_penalty_steps(int penalty, double lambda, double delta, uint64_t n, const double* alpha,
                        const double* beta, const float* x9, double* step);

// Synthetic raw data on the CPU (phantom.h), raw[Readings][n_ch][n_rows].
void port_synth(const ctbb_geom_c* geom, const ctbb_phantom_spec* spec, float* raw);

#ifdef __cplusplus
}
#endif
