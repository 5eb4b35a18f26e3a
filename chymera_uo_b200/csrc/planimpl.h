// planimpl.h -- the plan object behind the C ABI (internal to libchy_pot3).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <vector>

#include "chy_pot3.h"
#include "devplan.h"
#include "plan.h"

enum ChyStage { ST_FWD = 0, ST_BDY, ST_SYNTH, ST_SOLVE, ST_INV, ST_NSTAGE };

struct MixedState;   // k_mixed.cu

struct chy_plan {
    chy::HostPlan hp;
    chy::DevTables t{};
    int precision = CHY_PREC_FP64;
    int max_batch = 1;
    int refine = 1;
    int num_sms = 148;
    int device = 0;                // the device the plan's tables and work space live on
    // launch schedule (chy_autotune_multi picks these; 0 = the default)
    int mode_ctas = 0;             // persistent CTAs of the fused mixed mode solve (default: one per SM)
    int mode_kernel = 0;           // fused mixed mode solve: 0 auto, 1 one CTA per item, 2 CTA pairs (k_mode_pair)
    int blk_warps = 8;             // BLKTRI order: warps per CTA (4, 8, 16)
    int blk_ctas_per_sm = 2;       // BLKTRI order: CTAs per SM (blk_warps * this <= 16)
    int chunk = 0;                 // chy_solve_multi: solves per launch sequence (default max_batch)
    int streams = 0;               // chy_solve_multi: grids in flight at once (default 8)
    char *d_tables = nullptr;
    size_t table_bytes = 0;
    char *d_work = nullptr;
    size_t work_bytes = 0;
    chy::Work w{};
    size_t nvol = 0;
    // Host-pointer solves are staged through kStageSlots device slots of
    // stage_chunk solves each (RHO and PHI per solve), so the copy in of one
    // chunk, the solves of the next and the copy out of a third overlap.
    static constexpr int kStageSlots = 3;
    double *stage = nullptr;            // [slot][chunk][rho | phi] volumes
    size_t stage_bytes = 0;
    int stage_chunk = 0;
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
    cudaEvent_t ev_start = nullptr;
    cudaEvent_t ev_in[kStageSlots] = {}, ev_done[kStageSlots] = {}, ev_out[kStageSlots] = {};
    double *h_diag = nullptr;   // pinned
    double *coef_host = nullptr;   // /COEFS/ host destination (chy_plan_set_coef_host)
    double *coef_dev = nullptr;    // device COEF buffer owned by the plan
    size_t coef_bytes = 0;
    chy::StarDev star;             // ExternalPot (chy_plan_set_external, chy_plan_set_binary)
    double bin_a = 0.0;            // the BINARY companion's separation ABIN
    int last_slot = 0;             // batch slot of the latest solve launched
    bool profile = false;
    // One event set per profiled launch sequence, read back lazily (after
    // the caller has synchronised) so profiling adds no host waits.
    std::vector<std::array<cudaEvent_t, ST_NSTAGE + 1>> ev;
    size_t ev_used = 0;
    double stage_ms[ST_NSTAGE] = {};
    long long stage_calls = 0;
    long long launches = 0;
    MixedState *mx = nullptr;
};

// Host <-> device copies of host-pointer solves move whole arrays as single
// linear copies: with copies running in both directions at once, pitched (2-D)
// copies of the read and write sets reached about 12% less PCIe throughput on
// B200 hosts, and linear copies of sub-spans starting inside the array about
// 9% less, than linear copies of the whole (page-aligned) arrays.
//
// Copies one solve's PHI from device to the caller's host array, whole: the
// write set (PHI(1:JMAX+1, 1, :) and PHI(:, 2:KMAX+1, :)) and the cells a solve
// never writes (PHI(:, KMAX+2, :) and PHI(JMAX+2, 1, :)).  Those cells of the
// device copy hold the caller's own values, brought in earlier in the same call
// (by chy_internal_rim_in from pinned host memory, else by copy_phi_rim), so
// the host gets them back unchanged.
inline cudaError_t copy_phi_out(double *host, const double *dev, int J, int K, int L, cudaStream_t s)
{
    const size_t n = ((size_t)J + 2) * ((size_t)K + 2) * (size_t)L;
    return cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, s);
}

// Copies one solve's RHO from the caller's host array to the device, whole
// (a solve reads RHO(2:JMAX, 2:KMAX, :); the INDIRECT star shift also row
// KMAX+1; no kernel reads the other cells).
inline cudaError_t copy_rho_in(double *dev, const double *host, int J, int K, int L, cudaStream_t s)
{
    const size_t n = ((size_t)J + 2) * ((size_t)K + 2) * (size_t)L;
    return cudaMemcpyAsync(dev, host, n * sizeof(double), cudaMemcpyHostToDevice, s);
}

// Copies the cells of PHI that a solve never writes, PHI(:, KMAX+2, :) and
// PHI(JMAX+2, 1, :), between the caller's host array and a device copy (in
// either direction, by `kind`).  The external potential updates them in place.
inline cudaError_t copy_phi_rim(double *dst, const double *src, int J, int K, int L, cudaMemcpyKind kind,
                                cudaStream_t s)
{
    const size_t J2 = (size_t)J + 2, K2 = (size_t)K + 2, plane = J2 * K2 * sizeof(double);
    const size_t top = J2 * ((size_t)K + 1);
    cudaError_t e = cudaMemcpy2DAsync(dst + top, plane, src + top, plane, J2 * sizeof(double), L, kind, s);
    if (e != cudaSuccess) return e;
    return cudaMemcpy2DAsync(dst + J + 1, plane, src + J + 1, plane, sizeof(double), L, kind, s);
}

// The device-visible address of a caller's host array when it is pinned and
// mapped (cudaMallocHost / cudaHostAlloc memory under unified addressing),
// else nullptr (api.cu).
const double *chy_internal_mapped_view(const double *host);

// The cells of PHI a solve never writes, read by a kernel on `s` from the
// caller's mapped host array `src` (see chy_internal_mapped_view) into the
// device copy: the same cells copy_phi_rim moves, without the copy engine's
// hundreds of small row transfers per solve (api.cu).
cudaError_t chy_internal_rim_in(double *dev, const double *src, int J, int K, int L, cudaStream_t s);

// Sets the calling thread's chy_last_error message; returns code (api.cu).
int chy_internal_fail(int code, const char *msg);

// One launch sequence over nb device-pointer solves (api.cu).
int chy_internal_run_batch(chy_plan *p, const chy::BatchPtrs &bp, int nb, cudaStream_t s);

// Mixed-precision mode solve (k_mixed.cu).
bool chy_mixed_supported(const chy::HostPlan *hp);
// Appends the mixed path's tables to the packed table image; returns offset.
size_t chy_mixed_pack_tables(const chy::HostPlan *hp, std::vector<char> *image, bool mixed);
void chy_mixed_bind_tables(chy_plan *p, char *dev_base);
// Extra work-space doubles the mixed path needs (all batch slots).
size_t chy_mixed_work_doubles(const chy_plan *p);
void chy_mixed_bind_work(chy_plan *p, double *base);
// Solves the modes of nb solves in place in X; reports its launch count.
int chy_mixed_solve(chy_plan *p, int nb, cudaStream_t s, int *launches);
// After a stream sync: reads the device error word and the per-mode
// correction norms; CHY_ERR_TIMEOUT if a bounded wait expired.
int chy_mixed_collect(chy_plan *p, int nb);
void chy_mixed_fill_diag(const chy_plan *p, int slot, chy_diag *d);
// Enqueues on s a copy of the device error word into *host_word (pinned)
// and its reset; the word is non-zero after the stream is synchronised if a
// bounded wait of an earlier mode solve expired.  No-op for other paths.
int chy_mixed_read_error(chy_plan *p, int *host_word, cudaStream_t s);
// The plan's own pinned error word (mixed plans), else null.
int *chy_mixed_host_error_word(chy_plan *p);
// Test hook behind chy_dbg_mixed_probe.
// The kernel of the plan's last mixed mode solve: 0 none / not mixed, 1 k_mode_mixed,
// 2 k_mode_pair, 3 the wide pipeline.
int chy_mixed_last_kernel(const chy_plan *p);
int chy_dbg_mixed_probe_set(chy_plan *p, int polls);
// Allocates the FP64 iterate used when two or more corrections are set.
int chy_mixed_ensure_iterate(chy_plan *p);
size_t chy_mixed_iterate_bytes(const chy_plan *p);
void chy_mixed_release(chy_plan *p);
