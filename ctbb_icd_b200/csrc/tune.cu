// Autotuner for grouped ICD (no reference counterpart; the reference has one
// sequential order). Picks the number of concurrent voxel updates (warps in
// flight) and the tile edge of the visiting order by the measured decrease
// of the FP64 cost per millisecond of device time, probed from the current
// iterate; the iterate and error sinogram are restored afterwards.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gpu_internal.h"

using namespace ctbb;

extern "C" ctbb_status ctbb_gpu_recon_autotune(ctbb_recon* rc, const ctbb_ssm* ssm, const ctbb_icd_opts* base,
                                               int32_t probe_iters, ctbb_icd_opts* best, ctbb_tune_report* report) {
    clear_error();
    if (!rc || !ssm || !best) return fail(CTBB_ERR_INVALID_ARG, "null argument");
    if (probe_iters <= 0 || probe_iters > 100) return fail(CTBB_ERR_INVALID_ARG, "probe_iters must be in [1, 100]");
    ctbb_icd_opts o{};
    if (base) o = *base;
    o.mode = CTBB_ICD_GROUPED;
    o.priority = 0;
    const int wsel = o.weights ? o.weights : CTBB_SSM_FP32;
    if ((wsel == CTBB_SSM_FP32 && !ssm->d_w32) || (wsel == CTBB_SSM_FP16 && !ssm->d_w16))
        return fail(CTBB_ERR_INVALID_ARG, "requested weight format is not held by the matrix");
    o.weights = wsel;
    CTBB_CUDA(cudaSetDevice(rc->ctx->device));
    CTBB_TRY(recon_to_grouped(rc, ssm));
    CTBB_TRY(ctbb_gpu_recon_refresh_residual(rc, ssm));
    double c0 = 0.0;
    CTBB_TRY(cost_f64(rc, ssm, false, &c0));
    cudaStream_t st = rc->ctx->stream;
    float *d_xs = nullptr, *d_es = nullptr;
    CTBB_CUDA(cudaMalloc(&d_xs, rc->nvox * sizeof(float)));
    if (cudaMalloc(&d_es, rc->data_size * sizeof(float)) != cudaSuccess) {
        cudaFree(d_xs);
        return fail(CTBB_ERR_OOM, "autotune snapshot");
    }
    auto copy = [&](float* dst_x, const float* src_x, float* dst_e, const float* src_e) {
        cudaError_t e = cudaMemcpyAsync(dst_x, src_x, rc->nvox * sizeof(float), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dst_e, src_e, rc->data_size * sizeof(float), cudaMemcpyDeviceToDevice, st);
        return e;
    };
    ctbb_status status = CTBB_OK;
    if (copy(d_xs, rc->d_x32, d_es, rc->d_e32) != cudaSuccess) status = fail(CTBB_ERR_CUDA, "autotune snapshot copy");

    // Candidates (warps per voxel, warps in flight, entries per lane, tile
    // edge, column stage): the lockstep stack kernel; the shared-memory
    // staged kernel with 4 or 8 updates per SM; one warp per voxel streaming the column twice at
    // 1/4 .. 2 times the coupling-bound default; 8 or 16 entries per lane in
    // flight, the default tile edge for that concurrency (and half of it);
    // 4 or 8 warps per voxel with four or eight updates per SM. Launches cap the updates in
    // flight at the visiting order's bound, so candidates that collapse onto
    // the same effective shape run once.
    const int w0 = default_warps_in_flight(rc);
    const int sms = rc->ctx->sm_count;
    const int wmax = sms * 48;
    struct Cand {
        int wpv, w, epl, half, stage, pairs;  // pairs: entry_pairs (0 pairs with FP16, -1 single entries)
    };
    std::vector<Cand> cands;
    // Lockstep stacks: two CTAs of 16 updates per SM with 8 entries per lane
    // in flight. (One CTA with 16 entries per lane measured about twice as
    // slow on the 512 x 512 x 64 workload and is not probed.)
    cands.push_back({1, 2 * 16 * sms, 8, 0, 3, 0});
    // Shared-memory staged kernels: one CTA per SM with 4 (or 8) updates,
    // the matrix read once per update.
    for (int epl : {16, 8}) {
        cands.push_back({1, 4 * sms, epl, 0, 1, 0});
        cands.push_back({1, 8 * sms, epl, 0, 2, 0});
    }
    cands.push_back({1, 4 * sms, 16, 1, 1, 0});
    for (int epl : {8, 16})
        for (int m4 : {1, 2, 4, 8}) {
            const int w = std::max(32, std::min(wmax, w0 * m4 / 4));
            cands.push_back({1, w, epl, 0, 0, 0});
            if (m4 == 4 && epl == 8) cands.push_back({1, w, epl, 1, 0, 0});
            // the same shape over single entries (FP16 weights read as pairs above)
            if (m4 == 4 && epl == 16 && o.weights == CTBB_SSM_FP16) cands.push_back({1, w, epl, 0, 0, -1});
        }
    // Several warps per update (the column's entries, or entry pairs with
    // FP16 weights, kept in registers): four or eight updates per SM.
    cands.push_back({4, 4 * sms * 4, 8, 0, 0, 0});
    if (o.weights == CTBB_SSM_FP16) cands.push_back({4, 4 * sms * 4, 8, 0, 0, -1});
    cands.push_back({4, 8 * sms * 4, 8, 0, 0, 0});
    cands.push_back({8, 4 * sms * 8, 8, 0, 0, 0});
    // One update per CTA of 8 warps with the entry pairs bulk-copied into
    // shared memory: one stage (four CTAs per SM) or two (three per SM).
    // These kernels read entry pairs only: build them now (outside any
    // stream capture) and skip the kernels for a matrix whose detector-row
    // runs do not pair up (z flying focal spot), which keeps none.
    if (o.weights == CTBB_SSM_FP16 && status == CTBB_OK) status = ssm_build_pairs(const_cast<ctbb_ssm*>(ssm));
    if (o.weights == CTBB_SSM_FP16 && status == CTBB_OK && ssm->d_pairs) {
        cands.push_back({8, 4 * sms * 8, 8, 0, 4, 0});
        cands.push_back({8, 3 * sms * 8, 8, 0, 5, 0});
        // The one-stage kernel with the next item claimed during the
        // current update's penalty solve, four CTAs per SM.
        cands.push_back({8, 4 * sms * 8, 8, 0, 6, 0});
    }
    struct Trial {
        int wpv, w, epl, t, stage, pairs;
        double ms, cost, score;
    };
    std::vector<Trial> trials;
    int ibest = -1;
    for (const Cand& cd : cands) {
        {
            if (status != CTBB_OK || trials.size() >= CTBB_TUNE_MAX_TRIALS) break;
            ctbb_icd_opts c = o;
            c.warps_in_flight = cd.w;
            c.warps_per_voxel = cd.wpv;
            c.entries_per_lane = cd.epl;
            c.stage_column = cd.stage;
            c.entry_pairs = cd.pairs;
            c.lattice = 0;
            const int t_auto = lattice_spacing(rc, c);
            c.lattice = cd.half ? std::max(4, t_auto / 2) : t_auto;
            if (cd.half && c.lattice == t_auto) continue;
            const uint64_t bound = max_items_in_flight(rc->n_order ? rc->n_order : rc->nvox,
                                                       (int)rc->geom.num_voxels_z, c.lattice);
            // The claim-ahead bulk kernel holds two claimed items per CTA.
            const uint64_t items = std::max<uint64_t>(
                1, std::min<uint64_t>(requested_items(rc, c), cd.stage == 6 ? bound / 2 : bound));
            c.warps_in_flight = (int)(items * (uint64_t)cd.wpv);
            bool seen = false;
            for (const Trial& tr : trials)
                seen |= tr.wpv == c.warps_per_voxel && tr.w == c.warps_in_flight && tr.t == c.lattice &&
                        tr.epl == c.entries_per_lane && tr.stage == c.stage_column && tr.pairs == c.entry_pairs;
            if (seen) continue;
            if (copy(rc->d_x32, d_xs, rc->d_e32, d_es) != cudaSuccess) {
                status = fail(CTBB_ERR_CUDA, "autotune restore");
                break;
            }
            double ms_tot = 0.0;
            for (int i = 0; i < probe_iters && status == CTBB_OK; ++i) {
                float ms = 0.f;
                status = launch_icd_grouped(rc, ssm, c, &ms, nullptr, nullptr);
                ms_tot += ms;
            }
            if (status != CTBB_OK) break;
            status = ctbb_gpu_recon_refresh_residual(rc, ssm);
            double cost = 0.0;
            if (status == CTBB_OK) status = cost_f64(rc, ssm, false, &cost);
            if (status != CTBB_OK) break;
            const double score = (c0 - cost) / std::max(ms_tot, 1e-3);
            trials.push_back(
                {c.warps_per_voxel, c.warps_in_flight, c.entries_per_lane, c.lattice, c.stage_column, c.entry_pairs,
                 ms_tot, cost, score});
            if (ibest < 0 || score > trials[ibest].score) ibest = (int)trials.size() - 1;
        }
    }
    if (status == CTBB_OK && copy(rc->d_x32, d_xs, rc->d_e32, d_es) != cudaSuccess)
        status = fail(CTBB_ERR_CUDA, "autotune restore");
    if (status == CTBB_OK && cudaStreamSynchronize(st) != cudaSuccess) status = fail(CTBB_ERR_CUDA, "autotune sync");
    cudaFree(d_xs);
    cudaFree(d_es);
    if (status != CTBB_OK) return status;
    if (ibest < 0) return fail(CTBB_ERR_INVALID_ARG, "autotune ran no trial");
    *best = o;
    best->warps_in_flight = trials[ibest].w;
    best->warps_per_voxel = trials[ibest].wpv;
    best->entries_per_lane = trials[ibest].epl;
    best->stage_column = trials[ibest].stage;
    best->entry_pairs = trials[ibest].pairs;
    best->lattice = trials[ibest].t;
    if (report) {
        memset(report, 0, sizeof(*report));
        report->n_trials = (int32_t)trials.size();
        report->best = ibest;
        report->start_cost = c0;
        for (size_t i = 0; i < trials.size(); ++i) {
            report->trials[i].warps_in_flight = trials[i].w;
            report->trials[i].warps_per_voxel = trials[i].wpv;
            report->trials[i].entries_per_lane = trials[i].epl;
            report->trials[i].stage_column = trials[i].stage;
            report->trials[i].entry_pairs = trials[i].pairs;
            report->trials[i].lattice = trials[i].t;
            report->trials[i].device_ms = trials[i].ms;
            report->trials[i].cost = trials[i].cost;
            report->trials[i].score = trials[i].score;
        }
    }
    return CTBB_OK;
}
