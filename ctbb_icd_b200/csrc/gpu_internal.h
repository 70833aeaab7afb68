// Device-resident objects behind the opaque handles of the C ABI, and the
// internal launch functions shared between translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <vector>

#include "common.h"

#define CTBB_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t err__ = (call);                                                            \
        if (err__ != cudaSuccess)                                                              \
            return ::ctbb::fail(err__ == cudaErrorMemoryAllocation ? CTBB_ERR_OOM : CTBB_ERR_CUDA, \
                                "%s:%d %s: %s", __FILE__, __LINE__, #call,                     \
                                cudaGetErrorString(err__));                                    \
    } while (0)

#define CTBB_TRY(call)                        \
    do {                                      \
        ctbb_status st__ = (call);            \
        if (st__ != CTBB_OK) return st__;     \
    } while (0)

struct ctbb_ctx {
    // Objects (matrices, reconstructions, batches) created on this context;
    // ctbb_gpu_destroy defers the teardown until the last of them is freed.
    std::atomic<int> refs{0};
    std::atomic<bool> closing{false};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 148;
    size_t smem_per_block_optin = 0;
    // Reusable FP64 reduction scratch (partial sums), sized on demand.
    double* d_partials = nullptr;
    size_t partials_cap = 0;
    // Work-queue head for the grouped ICD kernel.
    unsigned long long* d_queue = nullptr;
    int* d_flags = nullptr;  // device-side error flags
};

// Stored system matrix: per voxel column c = i + nx*j, entries sorted by
// q = row + Nrows*(channel + n_channels*view). colptr[c] is the first entry of
// column c; vptr[c*(nvsm+1) + v] is the offset (relative to colptr[c]) of the
// first entry of SSM view v, so a view window [v0, v1) is one contiguous run.
struct ctbb_ssm {
    ctbb_ctx* ctx = nullptr;
    ctbb_geom_c geom{};
    uint64_t ncol = 0, nvsm = 0, nnz = 0, max_col_nnz = 0;
    int64_t* d_colptr = nullptr;  // [ncol + 1]
    uint32_t* d_vptr = nullptr;   // [ncol * (nvsm + 1)]
    int32_t* d_idx = nullptr;     // [nnz]
    float* d_w32 = nullptr;       // [nnz] (CTBB_SSM_FP32 held)
    __half* d_w16 = nullptr;      // [nnz] (CTBB_SSM_FP16 held)
    // Entry pairs (built on first use from idx + w16, ssm_build_pairs):
    // {q, w0 | w1 << 16} for two entries at consecutive sinogram indices,
    // w1 = 0 for a lone entry; same column / per-view offset layout.
    int64_t* d_pcolptr = nullptr;  // [ncol + 1]
    uint32_t* d_pvptr = nullptr;   // [ncol * (nvsm + 1)]
    uint2* d_pairs = nullptr;      // [npairs]
    uint64_t npairs = 0;
    bool pairs_checked = false;  // build tried (pairs kept only where they pay)
    int weights = 0;
    int ffs = 0;
    double build_ms = 0.0;
    uint64_t bytes = 0;
};

// Device-resident ICD state. The sequential (parity) mode keeps the image
// and the sinogram estimate y_hat = A x in FP64 like icd_iteration.cpp:47-48;
// the grouped mode keeps an FP32 image and the FP32 error sinogram e = y - A x.
struct ctbb_recon {
    ctbb_ctx* ctx = nullptr;
    ctbb_geom_c geom{};
    uint64_t nvox = 0, data_size = 0;
    std::vector<uint64_t> slice_indices;
    int32_t* d_start = nullptr;  // [nz] first data view of each slice's SSM window
    float* d_raw = nullptr;      // y
    double* d_x64 = nullptr;     // sequential-mode image
    double* d_est64 = nullptr;   // sequential-mode A x (FP64); also FP64 refresh accumulator
    float* d_x32 = nullptr;      // grouped-mode image
    float* d_e32 = nullptr;      // grouped-mode y - A x
    int rep = 0;                 // 0: x64/est64 current, 1: x32/e32 current
    // Sum over voxels inside the FOV of in-range matrix entries (cached per matrix).
    const ctbb_ssm* entries_ssm = nullptr;
    double entries = 0.0;
    // Grouped-mode visiting order: packed (column * nz + slice) per item,
    // built once per lattice spacing.
    uint32_t* d_order = nullptr;
    uint64_t n_order = 0;
    int order_P = 0;
    // Where each slice stack (same-parity slices of one cell) starts in the
    // order, n_stacks + 1 entries (the last is n_order).
    uint32_t* d_stacks = nullptr;
    uint64_t n_stacks = 0;
    // Learned warm start: per-voxel priority (size of the warm-start step)
    // and the visiting order restricted to the highest-priority voxels.
    float* d_prio = nullptr;
    uint32_t* d_prio_order = nullptr;
    uint64_t n_prio_order = 0;
    uint32_t* d_prio_stacks = nullptr;
    uint64_t n_prio_stacks = 0;
    int prio_P = 0;
    // Grouped iteration captured in a CUDA graph, and the launch it encodes.
    cudaGraphExec_t icd_graph = nullptr;
    std::vector<unsigned char> icd_graph_key;
};

struct ctbb_cnn;

namespace ctbb {

// Reference counting of a context by the objects created on it.
void ctx_retain(ctbb_ctx* ctx);
void ctx_release(ctbb_ctx* ctx);

ctbb_status ensure_partials(ctbb_ctx* ctx, size_t n);

// ssm.cu
ctbb_status ssm_validate_geometry(const ctbb_geom_c& g);
ctbb_status ssm_build_pairs(ctbb_ssm* s);

// recon.cu
ctbb_status recon_to_grouped(ctbb_recon* rc, const ctbb_ssm* ssm);
ctbb_status recon_to_sequential(ctbb_recon* rc, const ctbb_ssm* ssm);
ctbb_status forward_project_f64(ctbb_recon* rc, const ctbb_ssm* ssm, bool from_x32, double* d_out);
ctbb_status cost_f64(ctbb_recon* rc, const ctbb_ssm* ssm, bool exact, double* out);

// icd_seq.cu
ctbb_status launch_icd_sequential(ctbb_recon* rc, const ctbb_ssm* ssm, int n_iter, float* ms);

// icd_grouped.cu
ctbb_status launch_icd_grouped(ctbb_recon* rc, const ctbb_ssm* ssm, const ctbb_icd_opts& o,
                               float* ms, double* entries, uint64_t* items, double* scattered = nullptr);
int stage_capacity(const ctbb_ctx* ctx, int nw, int wbytes);
int default_warps_in_flight(const ctbb_recon* rc);
int lattice_spacing(const ctbb_recon* rc, const ctbb_icd_opts& o);
uint64_t requested_items(const ctbb_recon* rc, const ctbb_icd_opts& o);
uint64_t max_items_in_flight(uint64_t n_items, int nz, int T);
ctbb_status inrange_entries(ctbb_recon* rc, const ctbb_ssm* ssm, double* out);

// rotate.cu
ctbb_status rotate_volume(ctbb_ctx* ctx, const ctbb_geom_c& g, const double* tube_angles_deg,
                          const uint64_t* slice_indices, const float* d_in, float* d_out, int direction);

// cnn_tc.cu
ctbb_status conv_mid_tc(ctbb_ctx* ctx, int nx, int ny, int nz, const __nv_bfloat16* in, const __nv_bfloat16* wt,
                        const float* bias, const __nv_bfloat16* residual, const __nv_bfloat16* mask, int relu,
                        __nv_bfloat16* out, int* err);

// cnn.cu
ctbb_status cnn_predict_correction(ctbb_cnn* c, const float* x_dev, int nx, int ny, int nz, float* d_dev);
ctbb_status apply_correction(ctbb_ctx* ctx, uint64_t n, float* x_dev, const float* d_dev, float* prio_dev);
ctbb_ctx* cnn_ctx(const ctbb_cnn* c);
ctbb_status cnn_check_flag(ctbb_cnn* c);

}  // namespace ctbb
