// MD-coupled FEM (the reference's ms-stem-fem-md, src/ftem_lammps.cpp): every
// probe position is simulated through `samples` configurations of the
// specimen and its exit waves are averaged coherently (ftem_lammps.cpp:
// 1513-1540 sample loop, 2816-3287 slices and propagation, 3385-3402 ADF,
// 3403-3516 MTF, 3601-3610 accumulation, 3686-3990 FEM on the average).
//
// The reference rebuilds slices and transmission functions for every probe
// and sample.  Here the configurations are a fixed set of snapshot
// specimens, sample s using snapshot s mod n_snap, so each snapshot's
// slices are built once, stay resident, and serve every probe batch:
//
//   per batch of B probes, per sample s:
//     the 2 S_s fused slice passes over snapshot s (batched, split-wave
//     FP32 or FP64) -> ADF sum of this sample, added / samples (FP64)
//     -> [detector MTF] -> psi_acc += exit wave / samples (FP64)
//   then the FEM ring / cell / pixel sums of psi_acc, and the usual host
//   finish (ADF image = the sample-averaged ADF sums).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "engine.hpp"
#include "trace.hpp"
#include "kernels.h"

namespace msf {

namespace {

#define MSF_CUDA(call)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) +      \
                " at " + __FILE__ + ":" + std::to_string(__LINE__));        \
      return MSF_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)

#define MSF_TRY(call)                \
  do {                               \
    msf_status s_ = (call);          \
    if (s_ != MSF_OK) return s_;     \
  } while (0)

SegmentPlan segment_plan(const RasterPlan& P, double* partial) {
  SegmentPlan seg;
  seg.idx = P.seg_idx.as<int32_t>();
  seg.chunk_begin = P.chunk_begin.as<int32_t>();
  seg.seg_chunk = P.seg_chunk.as<int32_t>();
  seg.n_chunks = P.n_chunks;
  seg.ng = P.n_seg;
  seg.partial = partial;
  return seg;
}

bool same_cell(const Grid& a, const Grid& b) {
  return a.nx == b.nx && a.ny == b.ny && a.voltage == b.voltage && a.xperiod == b.xperiod &&
         a.yperiod == b.yperiod && a.xpd == b.xpd && a.ypd == b.ypd && a.xmin == b.xmin &&
         a.ymin == b.ymin;
}

}  // namespace

msf_status run_md(msf_context* ctx, int n_snap, const msf_specimen* const* snaps, int samples,
                  const msf_optics* optics, const msf_raster* raster, const msf_detect* det,
                  msf_results* res) {
  TraceScope trace_scope("md_raster");
  if (!ctx || !snaps || !optics || !raster || !det || !res) {
    set_error("null argument");
    return MSF_ERR_ARG;
  }
  if (n_snap < 1 || samples < 1 || samples % n_snap != 0) {
    set_error("MD samples (" + std::to_string(samples) + ") must be a positive multiple of the " +
              "number of snapshots (" + std::to_string(n_snap) +
              "), so that every probe sees the same sequence");
    return MSF_ERR_ARG;
  }
  for (int k = 0; k < n_snap; ++k) {
    if (!snaps[k] || snaps[k]->ctx != ctx) {
      set_error("snapshot specimen " + std::to_string(k) + " does not belong to this context");
      return MSF_ERR_ARG;
    }
    if (!same_cell(snaps[k]->g, snaps[0]->g)) {
      set_error("snapshot " + std::to_string(k) +
                " differs from the first in grid, voltage or lateral cell (x/y periods and "
                "minima must stay fixed)");
      return MSF_ERR_ARG;
    }
  }
  const bool fp64 = ctx->fp64;
  const size_t cbytes = fp64 ? 16 : 8;
  const Grid& g = snaps[0]->g;
  const int64_t plane = (int64_t)g.nx * g.ny;
  MSF_CUDA(cudaSetDevice(ctx->device));

  // per snapshot: probe, vacuum tables and shifts, detection of the ADF
  // annulus only; the full detection runs on the averaged waves (acc plan)
  msf_detect det_adf = *det;
  det_adf.outputs = MSF_OUT_ADF_IMAGE;
  det_adf.n_mtf = 0;
  std::vector<RasterPlan> plans(n_snap);
  for (int k = 0; k < n_snap; ++k)
    MSF_TRY(plan_raster(ctx, snaps[k], optics, raster, &det_adf, &plans[k]));
  RasterPlan A;
  MSF_TRY(plan_raster(ctx, snaps[0], optics, raster, det, &A));
  const int64_t n_probes = A.n_probes;
  const int n_seg = A.n_seg, n_k = A.n_k;

  // batch: the wavefields, their FP64 average and (MTF) the filtered waves
  int B = ctx->batch_for(g.nx, g.ny);
  if (B <= 0) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const int64_t per = (int64_t)(cbytes + 16 + (A.mtf ? 16 : 0)) * plane;
    B = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)(0.5 * (double)free_b) / per, 64));
  }
  B = (int)std::min<int64_t>(B, n_probes);
  int max_chunks = A.n_chunks;
  for (const auto& P : plans) max_chunks = std::max(max_chunks, P.n_chunks);
  DevBuf psi, acc, mtf_psi, partial, s_amp, s_int, adf_acc, d_err;
  MSF_TRY(ctx->alloc(&psi, cbytes * plane * B));
  MSF_TRY(ctx->alloc(&acc, 16 * plane * B));
  if (A.mtf) MSF_TRY(ctx->alloc(&mtf_psi, 16 * plane * B));
  MSF_TRY(ctx->alloc(&partial, sizeof(double) * 2 * B * std::max(max_chunks, 1)));
  MSF_TRY(ctx->alloc(&s_amp, sizeof(double) * B));
  MSF_TRY(ctx->alloc(&s_int, sizeof(double) * B));
  MSF_TRY(ctx->alloc(&adf_acc, sizeof(double) * B));
  MSF_TRY(ctx->alloc(&d_err, sizeof(int)));
  cudaStream_t st = ctx->stream;
  MSF_CUDA(cudaMemsetAsync(d_err.p, 0, sizeof(int), st));

  const bool pipe_col =
      pipe_supported(g.nx, g.ny, fp64) && (ctx->pipe_for(g.nx, g.ny) & MSF_PIPE_COL);
  alignas(64) unsigned char col_map[128];
  if (pipe_col) MSF_CUDA(encode_column_map(psi.p, B, g.nx, g.ny, col_map, fp64));
  PassArgs row, col;
  // columns the band limit removes entirely are skipped (same grid, hence
  // the same mask, for every snapshot)
  const bool skip_dead = pipe_col && snaps[0]->n_live_groups > 0;
  row.psi = col.psi = psi.p;
  row.batch_stride = col.batch_stride = plane;
  row.nx = col.nx = g.nx;
  row.ny = col.ny = g.ny;
  MSF_TRY(ctx->twiddles(g.ny, fp64, &row.tw));
  MSF_TRY(ctx->twiddles(g.nx, fp64, &col.tw));
  row.inv_s = col.inv_s = 1.0 / g.s;
  row.first_scale = g.nxny / g.s;
  const SegmentPlan seg_acc = segment_plan(A, partial.as<double>());

  cudaEvent_t ev0, ev1;
  MSF_CUDA(cudaEventCreate(&ev0));
  MSF_CUDA(cudaEventCreate(&ev1));
  MSF_CUDA(cudaEventRecord(ev0, st));
  int64_t launches = A.setup_launches, probe_slices = 0;
  for (const auto& P : plans) launches += P.setup_launches;
  for (int64_t p0 = 0; p0 < n_probes; p0 += B) {
    const int nb = (int)std::min<int64_t>(B, n_probes - p0);
    row.nb = col.nb = nb;
    MSF_CUDA(cudaMemsetAsync(acc.p, 0, 16 * plane * nb, st));
    MSF_CUDA(cudaMemsetAsync(adf_acc.p, 0, sizeof(double) * nb, st));
    for (int s = 0; s < samples; ++s) {
      const RasterPlan& P = plans[s % n_snap];
      const msf_specimen* spec = P.spec;
      const int S = P.S;
      const int32_t* shifts = P.d_shifts.as<int32_t>() + 2 * p0;
      row.shifts = shifts;
      row.probe = P.probe64.p;
      col.mask_lo = spec->mask_lo.as<int32_t>();
      col.mask_hi = spec->mask_hi.as<int32_t>();
      if (skip_dead) {
        row.row_dead_bits = spec->dead_bits.as<uint32_t>();
        col.live_groups = spec->live_groups.as<int32_t>();
        col.n_live_groups = spec->n_live_groups;
      }
      const char* tbase = static_cast<const char*>(spec->t.p);
      const char* pbase = static_cast<const char*>(spec->prop.p);
      const size_t prop_stride = cbytes * (g.nx + g.ny);
      for (int sl = 0; sl < S; ++sl) {
        row.trans = tbase + cbytes * plane * sl;
        row.row_dead_io = (sl > 0 ? 1 : 0) | (sl + 1 < S ? 2 : 0);
        RowOp op;
        if (fp64) {
          op = sl == 0 ? ROW_SLICE_FIRST : ROW_SLICE;
        } else {
          op = sl == 0 ? ROW_SPLIT_FIRST : ROW_SPLIT;
          row.psi0 = P.psi0_tab.as<float>() + 2 * plane * sl;
        }
        MSF_CUDA(launch_row(fp64, op, row, st));
        col.px = pbase + prop_stride * sl;
        col.py = pbase + prop_stride * sl + cbytes * g.nx;
        if (pipe_col)
          MSF_CUDA(launch_col_slice_pipe(col, sl + 1 == S, col_map, d_err.as<int>(), st, fp64));
        else
          MSF_CUDA(launch_col(fp64, sl + 1 == S ? COL_SLICE_LAST : COL_SLICE, col, st));
      }
      SplitK sk;
      if (!fp64) {
        sk.psi0k = P.psi0k.as<double>();
        sk.shifts = shifts;
        sk.nx = g.nx;
        sk.ny = g.ny;
      }
      // this sample's ADF signal (ftem_lammps.cpp:3385-3402): stem_image +=
      // detected intensity / samples
      MSF_CUDA(launch_segment_sums(fp64, psi.p, plane, nb, segment_plan(P, partial.as<double>()),
                                   s_amp.as<double>(), s_int.as<double>(), sk, st));
      MSF_CUDA(launch_strided_accumulate(adf_acc.as<double>(), 1, s_int.as<double>(), 1, nb,
                                         (double)samples, st));
      if (A.mtf) {  // ftem_lammps.cpp:3403-3516, then accumulated
        MSF_TRY(mtf_stage(ctx, A, fp64, psi.p, nb, sk, mtf_psi.as<double>(), st));
        MSF_CUDA(launch_wave_accumulate(true, mtf_psi.p, plane, nb, plane, SplitK{},
                                        (double)samples, acc.as<double>(), st));
      } else {
        MSF_CUDA(launch_wave_accumulate(fp64, psi.p, plane, nb, plane, sk, (double)samples,
                                        acc.as<double>(), st));
      }
      launches += 2 * S + 2 + 1 + 1 + (A.mtf ? 8 : 0);
      probe_slices += (int64_t)nb * S;
    }
    // FEM sums of the averaged waves (ftem_lammps.cpp:3686-3990); the ADF
    // column holds the sample-averaged ADF signal
    double* amp_out = A.amp.as<double>() + p0 * n_seg;
    double* int_out = A.inten.as<double>() + p0 * n_seg;
    MSF_CUDA(launch_segment_sums(true, acc.p, plane, nb, seg_acc, amp_out, int_out, SplitK{}, st));
    MSF_CUDA(cudaMemcpy2DAsync(int_out + n_k, sizeof(double) * n_seg, adf_acc.p, sizeof(double),
                               sizeof(double), nb, cudaMemcpyDeviceToDevice, st));
    launches += 2;
    if (A.pix_modes) {
      MSF_CUDA(launch_pixel_accum(true, acc.p, plane, nb, plane, A.acc_a.as<double>(),
                                  A.acc_i.as<double>(), SplitK{}, st));
      launches += 1;
    }
    if (p0 + nb == n_probes && res->final_psi) {
      // the last probe's averaged wave (ftem_lammps.cpp:4977-4990 "_final")
      MSF_CUDA(cudaMemcpyAsync(res->final_psi, acc.as<double>() + 2 * plane * (nb - 1),
                               16 * plane, cudaMemcpyDeviceToHost, st));
      ctx->d2h_bytes += 16 * plane;
    }
  }
  MSF_CUDA(cudaEventRecord(ev1, st));
  MSF_CUDA(cudaStreamSynchronize(st));
  int err_flag = 0;
  MSF_CUDA(cudaMemcpy(&err_flag, d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (err_flag) {
    set_error("a pipelined slice pass gave up waiting for a tile copy (bounded wait)");
    return MSF_ERR_TIMEOUT;
  }
  float ms = 0;
  MSF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  MSF_TRY(finish_raster(ctx, A, st, res));
  res->seconds_raster = 1e-3 * ms;
  res->seconds_setup = 0;
  res->probe_slices = probe_slices;
  res->kernel_launches = launches;
  return MSF_OK;
}

}  // namespace msf
