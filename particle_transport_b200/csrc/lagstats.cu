// Lag-pair statistics on the device.
//
// D_mumu / <dmu^2> (process_mu_chunk_dmumu_cpu!, src/compute_delta_mu2_dmumu_full.jl:457-704)
// -----------------------------------------------------------------------------------------
// Work unit = (particle, lag).  A warp owns one particle and 32 lags (lane =
// lag); all lanes therefore visit the same start save s at the same time, and
// the bin of a pair depends only on mu(s).  Each particle's mu series is
// staged on chip together with the list of its valid start saves sorted
// (stably) by start bin, so the pair loop runs bin by bin: every lane keeps
// (count, sum dmu, sum dmu^2) for the current bin in registers and flushes
// once per bin per particle into the CTA's shared (bin, lag) accumulators.
// Per-particle <dmu^2> values feed per-lane Welford triples in registers.
// CTA results go to per-CTA partials and a finalize kernel reduces them in
// CTA order, merging Welford triples with the reference formula
// (combine_welford_stats!, :439-455).  Integer counts are exact; FP64 sums
// differ from the reference only by summation order.
//
// D_pp (process_momenta_chunk_dpp_cpu!, src/compute_dpp_full.jl:247-288)
// ---------------------------------------------------------------------
// Same layout without bins: |p| is computed once per (particle, save) in FP64
// and every lane keeps its lag's count, sum(dp) and sum(dp^2) in registers for
// the whole launch; the normalised sums sum(dp/p0) = sum(dp)/p0 and
// sum((dp/p0)^2) = sum(dp^2)/p0^2 are formed once per lag at the end, which
// equals the reference's per-pair division up to rounding.
#include <math_constants.h>

#include "exact_mu.cuh"

#include <cstdlib>
#include <cstring>
#include "pt_internal.cuh"

#include <algorithm>

namespace pt {
namespace {

constexpr int kWarp = 32;
constexpr int kStageWarps = 8;  // warps of a particle slot that stage its series

struct WelfordPart {
    long long count;
    double mean, m2, pair_ss;
    long long pair_n;
};

// combine_welford_stats! (src/compute_delta_mu2_dmumu_full.jl:439-455)
__device__ __forceinline__ void welford_merge(long long& gc, double& gm, double& gm2, long long lc, double lm,
                                              double lm2)
{
    if (lc <= 0) return;
    if (gc == 0) {
        gc = lc; gm = lm; gm2 = lm2;
        return;
    }
    long long cc = gc + lc;
    double delta = lm - gm;
    gm += delta * (double)lc / (double)cc;
    gm2 += lm2 + delta * delta * (double)gc * (double)lc / (double)cc;
    gc = cc;
}

// mu_bin_value + mu_bin_index_full (dmumu:304-318): 0-based bin, n_bins for a
// finite value outside [edges[0], edges[n_bins]], -1 for a non-finite value.
// searchsortedlast (the last edge <= v) is found from a guess on a uniform
// grid, inv_w = n_bins / (edges[n_bins] - edges[0]), moved up and down until
// edges[b] <= v < edges[b + 1]: the same bin as a binary search over the
// stored Float64 edges for any increasing edges, in one or two compares for
// the uniform edges of build_mu_edges_full (a range).
__device__ __forceinline__ int bin_of(double v, const double* __restrict__ edges, int n_bins, int bin_abs,
                                      double inv_w)
{
    if (!isfinite(v)) return -1;
    if (bin_abs) v = fabs(v);
    if (v < edges[0] || v > edges[n_bins]) return n_bins;
    int b = (int)fmin(fmax((v - edges[0]) * inv_w, 0.0), (double)(n_bins - 1));
    while (b < n_bins && edges[b + 1] <= v) ++b;
    while (b > 0 && edges[b] > v) --b;
    return b == n_bins ? n_bins - 1 : b;  // v == edges[n_bins] falls in the last bin
}

struct DmumuLaunch {
    int64_t n, nsave;
    int64_t start_cap;         // 1 for the injection estimator, nsave for sliding
    const int64_t* lags;       // this batch's lags
    int nl;                    // lags in this batch
    const double* edges;
    int n_bins, bin_abs;
    int ppc, groups;           // particle slots per CTA, 32-lag groups per slot
    int parts;                 // warps splitting the bins of one (slot, lag group)
    size_t slot_bytes;
    char* gslots;              // global staging when the slots do not fit on chip
    // per-CTA outputs
    unsigned long long* part_cnt;  // [grid][nl][n_bins]
    double* part_sd;
    double* part_sd2;
    WelfordPart* part_w;           // [grid][nl]
};

// Where dmumu_kernel reads the mu series of particle p: a mu chunk at the
// compute precision T (the reference's mu_chunk, Float32 by default), element
// (p, s) at p * sp + s * ss.
template <typename T_>
struct CacheSourceT {
    using T = T_;
    const T_* mu;
    int64_t sp, ss;
    __device__ __forceinline__ T_ operator()(int64_t p, int64_t s) const { return mu[p * sp + s * ss]; }
};
using CacheSource = CacheSourceT<float>;
// bytes of one particle slot of dmumu_kernel (layout in the kernel)
size_t dmumu_slot_bytes(int64_t nsave, size_t mu_bytes, size_t idx_bytes, int n_bins, int nl_cap)
{
    auto a16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
    return a16((size_t)(nsave + 1) * mu_bytes) + a16((size_t)nsave * idx_bytes) +
           a16(sizeof(int) * (size_t)(kStageWarps * (n_bins + 1) + n_bins + 2)) + a16(16 * (size_t)nl_cap);
}

template <typename IdxT, bool SMEM_SLOTS, class Src>
__global__ void __launch_bounds__(1024) dmumu_kernel(DmumuLaunch a, Src source)
{
    using MuT = typename Src::T;
    extern __shared__ __align__(16) unsigned char smem[];
    const int nb = a.n_bins, nl = a.nl;
    // shared layout: edges | acc_cnt | acc_sd | acc_sd2 ([bin][lag] each) | slots
    double* s_edges = (double*)smem;
    size_t off = ((size_t)(nb + 1) * sizeof(double) + 15) & ~(size_t)15;
    unsigned long long* acc_cnt = (unsigned long long*)(smem + off);
    off += (size_t)nl * nb * sizeof(unsigned long long);
    double* acc_sd = (double*)(smem + off);
    off += (size_t)nl * nb * sizeof(double);
    double* acc_sd2 = (double*)(smem + off);
    off += (size_t)nl * nb * sizeof(double);
    unsigned char* slot_base = SMEM_SLOTS ? (smem + off) : (unsigned char*)(a.gslots + (size_t)blockIdx.x * a.ppc * a.slot_bytes);

    for (int i = threadIdx.x; i <= nb; i += blockDim.x) s_edges[i] = a.edges[i];
    const double span = a.edges[nb] - a.edges[0];
    const double inv_w = span > 0.0 && isfinite(span) ? (double)nb / span : 0.0;
    for (int i = threadIdx.x; i < nl * nb; i += blockDim.x) {
        acc_cnt[i] = 0ull;
        acc_sd[i] = 0.0;
        acc_sd2[i] = 0.0;
    }

    // Lags are dealt to the 32-lane groups so that lags equal modulo 32 --
    // which read the same shared-memory bank at every start -- fall into
    // different groups where possible.  s_lane_lag[g*32 + lane] = lag index
    // (-1: idle lane), s_lag_pos[lag] = g*32 + lane.
    __shared__ int s_lane_lag[8 * kWarp];
    __shared__ int s_lag_pos[8 * kWarp];
    __shared__ unsigned char cnt[8][kWarp];
    __shared__ int fill[8];
    for (int i = threadIdx.x; i < 8 * kWarp; i += blockDim.x) {
        s_lane_lag[i] = -1;
        cnt[i / kWarp][i % kWarp] = 0;
    }
    if (threadIdx.x < 8) fill[threadIdx.x] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < nl; ++i) {
            const int r = (int)(((a.lags[i] % kWarp) + kWarp) % kWarp);
            int best = -1;
            for (int g = 0; g < a.groups; ++g) {
                if (fill[g] >= kWarp) continue;
                if (best < 0 || cnt[g][r] < cnt[best][r] || (cnt[g][r] == cnt[best][r] && fill[g] < fill[best]))
                    best = g;
            }
            const int pos = best * kWarp + fill[best]++;
            cnt[best][r]++;
            s_lane_lag[pos] = i;
            s_lag_pos[i] = pos;
        }
    }
    __syncthreads();

    const int warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const int wps = a.groups * a.parts;  // warps per particle slot
    const int slot = warp / wps, group = (warp % wps) / a.parts, part = warp % a.parts;
    const int li = s_lane_lag[group * kWarp + lane];
    const bool lane_on = li >= 0;
    int64_t L = lane_on ? a.lags[li] : 0;
    if (L < 1 || L >= a.nsave) L = a.nsave;  // reference: lag >= nsteps -> skipped (valid starts: s < nsave - L)

    // slot layout: series[nsave + 1] MuT | list[nsave] IdxT | whist[kStageWarps][nb+1] int
    //              | cur[nb+2] int | tot_c[nl] u64 | tot_sd2[nl] f64 (per-particle totals over the bins)
    // The series holds the finite mu values and NaN for the others, and
    // series[nsave] = NaN: a lag partner past the end of the series reads it.
    unsigned char* sb = slot_base + (size_t)slot * a.slot_bytes;
    MuT* series = (MuT*)sb;
    IdxT* list = (IdxT*)(sb + (((a.nsave + 1) * sizeof(MuT) + 15) & ~(size_t)15));
    int* whist = (int*)((unsigned char*)list + ((a.nsave * sizeof(IdxT) + 15) & ~(size_t)15));
    int* cur = whist + kStageWarps * (nb + 1);
    unsigned long long* tot_c = (unsigned long long*)((unsigned char*)whist +
                                                      ((sizeof(int) * (size_t)(kStageWarps * (nb + 1) + nb + 2) + 15) &
                                                       ~(size_t)15));
    double* tot_sd2 = (double*)(tot_c + nl);
    // staging is shared by the first `stagers` warps of the slot, each taking a
    // contiguous range of saves; per-warp bin counts, offset in warp order,
    // give the same bin-sorted start list (ascending starts within a bin)
    // as a single warp walking the series
    const int wis = warp % wps;
    const int stagers = min(wps, kStageWarps);

    long long wc = 0, pn = 0;
    double wm = 0.0, wm2 = 0.0, pss = 0.0;
    const int64_t scap = min(a.start_cap, a.nsave);
    const unsigned lt_mask = (1u << lane) - 1u;

    __syncthreads();
    const int64_t tiles = (a.n + a.ppc - 1) / a.ppc;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t p = tile * a.ppc + slot;
        const bool have = p < a.n;
        // ---- stage: series, per-warp bin counts
        if (have && wis < stagers) {
            const int64_t per = ((a.nsave + stagers - 1) / stagers + kWarp - 1) / kWarp * kWarp;
            const int64_t st_begin = (int64_t)wis * per, st_end = min(a.nsave, st_begin + per);
            int* my_hist = whist + wis * (nb + 1);
            for (int b = lane; b <= nb; b += kWarp) my_hist[b] = 0;
            if (wis == 0) {
                for (int l = lane; l < nl; l += kWarp) {
                    tot_c[l] = 0ull;
                    tot_sd2[l] = 0.0;
                }
                if (lane == 0) series[a.nsave] = MuT(NAN);
            }
            __syncwarp();
            for (int64_t s0 = st_begin; s0 < st_end; s0 += kWarp) {
                const int64_t s = s0 + lane;
                int b = -1;
                if (s < st_end) {
                    const MuT v = source(p, s);
                    series[s] = isfinite(v) ? v : MuT(NAN);
                    if (s < scap) b = bin_of((double)v, s_edges, nb, a.bin_abs, inv_w);
                }
                const unsigned active = __ballot_sync(0xffffffffu, b >= 0);
                if (b >= 0) {
                    const unsigned same = __match_any_sync(active, b);
                    if ((same & lt_mask) == 0) my_hist[b] += __popc(same);
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // ---- offsets: bin-major, then stager order within a bin
        if (have && wis == 0) {
            int carry = 0;
            for (int b0 = 0; b0 <= nb; b0 += kWarp) {
                const int b = b0 + lane;
                int t = 0;
                if (b <= nb)
                    for (int w = 0; w < stagers; ++w) t += whist[w * (nb + 1) + b];
                int incl = t;
                for (int d = 1; d < kWarp; d <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, d);
                    if (lane >= d) incl += y;
                }
                if (b <= nb) {
                    int run = carry + incl - t;
                    cur[b] = run;
                    for (int w = 0; w < stagers; ++w) {
                        const int c = whist[w * (nb + 1) + b];
                        whist[w * (nb + 1) + b] = run;
                        run += c;
                    }
                }
                carry += __shfl_sync(0xffffffffu, incl, kWarp - 1);
            }
            if (lane == 0) cur[nb + 1] = carry;
        }
        __syncthreads();
        // ---- scatter each stager's starts in order
        if (have && wis < stagers) {
            const int64_t per = ((a.nsave + stagers - 1) / stagers + kWarp - 1) / kWarp * kWarp;
            const int64_t st_begin = (int64_t)wis * per, st_end = min(a.nsave, st_begin + per);
            int* my_hist = whist + wis * (nb + 1);
            const int64_t end = min(st_end, scap);
            for (int64_t s0 = st_begin; s0 < end; s0 += kWarp) {
                const int64_t s = s0 + lane;
                int b = -1;
                if (s < end) b = bin_of((double)series[s], s_edges, nb, a.bin_abs, inv_w);
                const unsigned active = __ballot_sync(0xffffffffu, b >= 0);
                if (b >= 0) {
                    const unsigned same = __match_any_sync(active, b);
                    const int rank = __popc(same & lt_mask);
                    list[my_hist[b] + rank] = (IdxT)s;
                    __syncwarp(active);
                    if (rank == 0) my_hist[b] += __popc(same);
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // ---- pairs: the `parts` warps of a (slot, lag group) split the
        // bin-sorted start list into equal shares (a bin may straddle two
        // shares; each flushes its part of it), so they reach the barrier
        // together whatever the particle's bin counts; every lane keeps two
        // accumulator chains
        if (have) {
            long long my_c = 0;
            double my_sd2 = 0.0;
            // starts, lags and nsave fit 32 bits (nsave < 2^31); so does a bin's count
            const unsigned n32 = (unsigned)a.nsave, L32 = (unsigned)L;
            const int total = cur[nb + 1];
            const int r0 = (int)(((long long)total * part) / a.parts);
            const int r1 = (int)(((long long)total * (part + 1)) / a.parts);
            int b = 0;
            if (r0 < r1)
                while (cur[b + 1] <= r0) ++b;  // the bin holding entry r0 (r0 < total = cur[nb + 1])
            for (int e = r0; e < r1; ++b) {
                const int e1 = min(cur[b + 1], r1);
                int c = 0;
                double sd0 = 0.0, sd1 = 0.0, sq0 = 0.0, sq1 = 0.0;
                // Branch-free pairs.  A start in the list has a finite mu; its
                // partner series[s + L] is NaN when the particle's mu is not
                // finite there, and s + L past the series end reads the NaN pad
                // (idle lanes have L = nsave).  An invalid partner is replaced by
                // the start's own value, so the pair adds +0 and 0 * 0 -- the
                // sums are bit-identical to skipping it (they are never -0).
                for (; e + 4 <= e1; e += 4) {
                    MuT a_[4], v_[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const unsigned s = (unsigned)list[e + k];
                        a_[k] = series[s];
                        v_[k] = series[min(s + L32, n32)];
                    }
#pragma unroll
                    for (int k = 0; k < 4; k += 2) {
                        const bool ok0 = v_[k] == v_[k], ok1 = v_[k + 1] == v_[k + 1];
                        const MuT w0 = ok0 ? v_[k] : a_[k], w1 = ok1 ? v_[k + 1] : a_[k + 1];
                        c += (int)ok0 + (int)ok1;
                        const double d0 = (double)w0 - (double)a_[k];
                        const double d1 = (double)w1 - (double)a_[k + 1];
                        sd0 += d0;
                        sq0 = fma(d0, d0, sq0);
                        sd1 += d1;
                        sq1 = fma(d1, d1, sq1);
                    }
                }
                for (; e < e1; ++e) {
                    const unsigned s = (unsigned)list[e];
                    const MuT av = series[s];
                    const MuT vv = series[min(s + L32, n32)];
                    const bool ok = vv == vv;
                    const double d = (double)(ok ? vv : av) - (double)av;
                    c += (int)ok;
                    sd0 += d;
                    sq0 = fma(d, d, sq0);
                }
                const double sd = sd0 + sd1, sd2 = sq0 + sq1;
                if (b < nb && c > 0 && lane_on) {
                    const int ai = b * nl + li;  // [bin][lag]: the lanes of a flush hit consecutive words
                    atomicAdd(&acc_cnt[ai], (unsigned long long)c);
                    atomicAdd(&acc_sd[ai], sd);
                    atomicAdd(&acc_sd2[ai], sd2);
                }
                my_c += c;
                my_sd2 += sd2;
                e = e1;
            }
            if (lane_on && my_c > 0) {
                atomicAdd(&tot_c[li], (unsigned long long)my_c);
                atomicAdd(&tot_sd2[li], my_sd2);
            }
        }
        __syncthreads();
        if (have && part == 0 && lane_on) {
            const long long tc = (long long)tot_c[li];
            const double ts = tot_sd2[li];
            if (tc > 0) {
                // per-particle value: mean dmu^2 over its valid pairs (dmumu:528-537);
                // for the injection estimator tc == 1 and the value is dmu^2 (:625-631)
                const double value = ts / (double)tc;
                wc += 1;
                const double delta = value - wm;
                wm += delta / (double)wc;
                wm2 += delta * (value - wm);
                pss += ts;
                pn += tc;
            }
        }
        __syncthreads();
    }

    // ---- CTA epilogue: (bin, lag) accumulators and Welford triples
    const int64_t cta = blockIdx.x;
    for (int i = threadIdx.x; i < nl * nb; i += blockDim.x) {
        const int j = (i % nb) * nl + i / nb;  // partials are [lag][bin], the shared sums [bin][lag]
        a.part_cnt[cta * nl * nb + i] = acc_cnt[j];
        a.part_sd[cta * nl * nb + i] = acc_sd[j];
        a.part_sd2[cta * nl * nb + i] = acc_sd2[j];
    }
    __syncthreads();
    // reuse the accumulator region to gather per-warp Welford triples
    WelfordPart* wp = (WelfordPart*)(smem + (((size_t)(nb + 1) * sizeof(double) + 15) & ~(size_t)15));
    const int nwarps = blockDim.x / kWarp;
    wp[warp * kWarp + lane] = WelfordPart{wc, wm, wm2, pss, pn};
    __syncthreads();
    for (int l = threadIdx.x; l < nl; l += blockDim.x) {
        const int g = s_lag_pos[l] / kWarp, ln = s_lag_pos[l] % kWarp;
        long long c = 0, n2 = 0;
        double m = 0.0, m2 = 0.0, ss = 0.0;
        for (int sl = 0; sl < a.ppc; ++sl) {
            const int w = sl * wps + g * a.parts;  // the part-0 warp holds the slot's Welford triple
            if (w >= nwarps) break;
            const WelfordPart q = wp[w * kWarp + ln];
            welford_merge(c, m, m2, q.count, q.mean, q.m2);
            ss += q.pair_ss;
            n2 += q.pair_n;
        }
        a.part_w[cta * nl + l] = WelfordPart{c, m, m2, ss, n2};
    }
}

// Reduce per-CTA partials in CTA order and add / merge into the outputs.
__global__ void dmumu_finalize_kernel(const unsigned long long* __restrict__ part_cnt,
                                      const double* __restrict__ part_sd, const double* __restrict__ part_sd2,
                                      const WelfordPart* __restrict__ part_w, int grid, int nl, int nb, int lag0,
                                      int n_lags_total, int64_t* counts, double* sum_d, double* sum_d2,
                                      int64_t* w_count, double* w_mean, double* w_m2, double* pair_ss,
                                      int64_t* pair_n)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nl * nb) {
        unsigned long long c = 0;
        double sd = 0.0, sd2 = 0.0;
        for (int g = 0; g < grid; ++g) {
            c += part_cnt[(int64_t)g * nl * nb + t];
            sd += part_sd[(int64_t)g * nl * nb + t];
            sd2 += part_sd2[(int64_t)g * nl * nb + t];
        }
        const int l = t / nb, b = t % nb;
        const int64_t o = (int64_t)(lag0 + l) * nb + b;  // Julia (n_bins, n_lags)
        counts[o] += (int64_t)c;
        sum_d[o] += sd;
        sum_d2[o] += sd2;
    }
    if (t < nl) {
        long long c = 0, n2 = 0;
        double m = 0.0, m2 = 0.0, ss = 0.0;
        for (int g = 0; g < grid; ++g) {
            const WelfordPart q = part_w[(int64_t)g * nl + t];
            welford_merge(c, m, m2, q.count, q.mean, q.m2);
            ss += q.pair_ss;
            n2 += q.pair_n;
        }
        const int l = lag0 + t;
        long long gc = w_count[l];
        double gm = w_mean[l], gm2 = w_m2[l];
        welford_merge(gc, gm, gm2, c, m, m2);
        w_count[l] = gc;
        w_mean[l] = gm;
        w_m2[l] = gm2;
        pair_ss[l] += ss;
        pair_n[l] += n2;
    }
    (void)n_lags_total;
}

// ------------------------------------------------------------------ D_pp
// momentum_magnitude (src/compute_dpp_full.jl:232-234) with the reference's
// rounding: explicitly rounded products and sums are never contracted into
// FMA, so |p| is bit-identical to the reference's and dp = p_end - p_start
// keeps its last bits.
__device__ __forceinline__ double pmag_exact(float px, float py, float pz)
{
    const double x = (double)px, y = (double)py, z = (double)pz;
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

struct DppPart {
    long long count;
    double sdp, sdp2;
};

struct DppLaunch {
    const float* mom;
    int64_t chunk, nsave;
    const int64_t* lags;
    int nl;
    double p0;
    int ppc, wps;  // particle slots per CTA, warps per slot
    size_t slot_bytes;
    char* gslots;
    DppPart* part;  // [grid][nl]
};

// Warps = (particle slot, lag subset): warp w of a slot owns lags w, w + wps,
// w + 2 wps, ... and takes kDppLags of them at a time; its lanes take the
// starts s = lane, lane + 32, ...  A warp's 8-byte |p| reads are then
// consecutive (no shared-memory bank conflicts, whatever the lags), and
// |p|[s] is read once for the lags of a pass.  The series of a slot holds |p| at saves 0..nsave-1 and
// NaN at index nsave, so the end of a pair past the series reads NaN (an
// invalid pair) with no bounds test.  A lag's sums are warp-reduced once per
// particle and added by lane 0 into the slot's accumulator for that lag (one
// writer per (slot, lag)); the CTA adds its slots in slot order at the end.
// lags of a warp per pass over the starts (|p|[s] read once for them); 4 was
// measured slower: a pass runs to the range of its smallest lag
constexpr int kDppLags = 2;

template <bool SMEM_SLOTS>
__global__ void __launch_bounds__(1024) dpp_kernel(DppLaunch a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    // shared layout: acc[ppc][nl] | slots (when on chip)
    DppPart* acc = (DppPart*)smem;
    const size_t acc_bytes = ((size_t)a.ppc * a.nl * sizeof(DppPart) + 15) & ~(size_t)15;
    unsigned char* slot_base =
        SMEM_SLOTS ? smem + acc_bytes : (unsigned char*)(a.gslots + (size_t)blockIdx.x * a.ppc * a.slot_bytes);
    for (int i = threadIdx.x; i < a.ppc * a.nl; i += blockDim.x) acc[i] = DppPart{0, 0.0, 0.0};
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const int slot = warp / a.wps, w = warp % a.wps;
    const int nsave = (int)a.nsave;  // nsave < 2^31
    double* series = (double*)(slot_base + (size_t)slot * a.slot_bytes);
    const int64_t tiles = (a.chunk + a.ppc - 1) / a.ppc;
    __syncthreads();
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        // cooperative staging: thread t -> (save, particle slot)
        const int64_t p0i = tile * a.ppc;
        const int np = (int)(a.chunk - p0i < (int64_t)a.ppc ? a.chunk - p0i : (int64_t)a.ppc);
        for (int64_t t = threadIdx.x; t < (int64_t)np * (a.nsave + 1); t += blockDim.x) {
            const int sl = (int)(t % np);
            const int64_t s = t / np;
            double v = CUDART_NAN;  // the pad at index nsave
            if (s < a.nsave) {
                const float* m = a.mom + s * 3 * a.chunk + p0i + sl;
                v = pmag_exact(m[0], m[a.chunk], m[2 * a.chunk]);
            }
            ((double*)(slot_base + (size_t)sl * a.slot_bytes))[s] = v;
        }
        __syncthreads();
        if (slot < np) {
            // |p| >= 0 or NaN or +inf, so pe - ps is finite exactly when both
            // ends are finite; an invalid pair adds 0 (branch-free), which
            // leaves the sums unchanged.  The normalised sums are sum(d)/p0
            // and sum(d^2)/p0^2, formed once per lag in dpp_finalize_kernel.
            for (int l0 = w; l0 < a.nl; l0 += kDppLags * a.wps) {
                int L[kDppLags], cnt[kDppLags];
                double sd[kDppLags], sq[kDppLags];
                int lmin = nsave;
#pragma unroll
                for (int k = 0; k < kDppLags; ++k) {
                    const int l = l0 + k * a.wps;
                    // the range test in 64 bits, before the narrowing
                    const int64_t v64 = l < a.nl ? a.lags[l] : a.nsave;
                    const int v = (v64 < 1 || v64 >= a.nsave) ? nsave : (int)v64;  // lag >= nsteps -> skipped
                    L[k] = v;
                    lmin = min(lmin, v);
                    cnt[k] = 0;
                    sd[k] = 0.0;
                    sq[k] = 0.0;
                }
                const int lim = nsave - lmin;
                for (int s = lane; s < lim; s += kWarp) {
                    const double ps = series[s];
#pragma unroll
                    for (int k = 0; k < kDppLags; ++k) {
                        const double pe = series[min((unsigned)s + (unsigned)L[k], (unsigned)nsave)];
                        double d = pe - ps;
                        const bool ok = isfinite(d);
                        d = ok ? d : 0.0;
                        cnt[k] += (int)ok;
                        sd[k] += d;
                        sq[k] = fma(d, d, sq[k]);
                    }
                }
#pragma unroll
                for (int k = 0; k < kDppLags; ++k) {
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        cnt[k] += __shfl_xor_sync(0xffffffffu, cnt[k], o);
                        sd[k] += __shfl_xor_sync(0xffffffffu, sd[k], o);
                        sq[k] += __shfl_xor_sync(0xffffffffu, sq[k], o);
                    }
                    const int l = l0 + k * a.wps;
                    if (lane == 0 && l < a.nl) {
                        DppPart& A = acc[slot * a.nl + l];
                        A.count += cnt[k]; A.sdp += sd[k]; A.sdp2 += sq[k];
                    }
                }
            }
        }
        __syncthreads();
    }
    // CTA epilogue: slots added in slot order
    for (int l = threadIdx.x; l < a.nl; l += blockDim.x) {
        DppPart r{0, 0, 0};
        for (int sl = 0; sl < a.ppc; ++sl) {
            const DppPart v = acc[sl * a.nl + l];
            r.count += v.count; r.sdp += v.sdp; r.sdp2 += v.sdp2;
        }
        a.part[(int64_t)blockIdx.x * a.nl + l] = r;
    }
}

__global__ void dpp_finalize_kernel(const DppPart* __restrict__ part, int grid, int nl, int lag0, double p0,
                                    int64_t* counts, double* sdp, double* sdp2, double* sdn, double* sdn2)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nl) return;
    DppPart r{0, 0, 0};
    for (int g = 0; g < grid; ++g) {
        const DppPart q = part[(int64_t)g * nl + t];
        r.count += q.count; r.sdp += q.sdp; r.sdp2 += q.sdp2;
    }
    const int l = lag0 + t;
    counts[l] += r.count;
    sdp[l] += r.sdp;
    sdp2[l] += r.sdp2;
    sdn[l] += r.sdp / p0;
    sdn2[l] += r.sdp2 / p0 / p0;
}

// ------------------------------------------------------------------ energies
// kinetic_energy_gev_from_pmag (dpp:236-240)
__device__ __forceinline__ double kinetic_gev(double pmag)
{
    if (!isfinite(pmag)) return NAN;
    const double gev_to_j = 1.0e9 * 1.602176634e-19;
    const double r = __ddiv_rn(pmag, M_P * C_LIGHT);
    const double gamma = __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(r, r)));
    return __ddiv_rn(__dmul_rn(__dmul_rn(__dadd_rn(gamma, -1.0), M_P), C_LIGHT * C_LIGHT), gev_to_j);
}

// snapshot indices outside [0, nsave) (possible for the device entry point,
// whose indices the host cannot see) give NaN instead of a stray read
__global__ void energy_snap_kernel(const float* __restrict__ mom, int64_t chunk, int64_t nsave,
                                   const int64_t* __restrict__ snaps, int n_snap, int64_t offset,
                                   double* __restrict__ out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= chunk * n_snap) return;
    const int64_t p = t % chunk;
    const int j = (int)(t / chunk);
    const int64_t sj = snaps[j];
    if (sj < 0 || sj >= nsave) {
        out[(offset + p) * n_snap + j] = NAN;
        return;
    }
    const float* m = mom + sj * 3 * chunk + p;
    out[(offset + p) * n_snap + j] = kinetic_gev(pmag_exact(m[0], m[chunk], m[2 * chunk]));
}

__global__ void energy_hist_kernel(const float* __restrict__ mom, int64_t chunk, int64_t nsave,
                                   const int64_t* __restrict__ snaps, int n_snap, double log_emin, double inv_dlog,
                                   int n_hist, unsigned long long* __restrict__ counts)
{
    extern __shared__ unsigned long long h[];
    for (int i = threadIdx.x; i < n_snap * n_hist; i += blockDim.x) h[i] = 0ull;
    __syncthreads();
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < chunk * n_snap;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = t % chunk;
        const int j = (int)(t / chunk);
        const int64_t sj = snaps[j];
        if (sj < 0 || sj >= nsave) continue;  // not a save of this chunk: counted nowhere
        const float* m = mom + sj * 3 * chunk + p;
        const double e = kinetic_gev(pmag_exact(m[0], m[chunk], m[2 * chunk]));
        if (!(e > 0.0) || !isfinite(e)) continue;
        const double f = (log(e) - log_emin) * inv_dlog;
        if (!(f >= 0.0) || f >= (double)n_hist) continue;
        atomicAdd(&h[j * n_hist + (int)f], 1ull);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_snap * n_hist; i += blockDim.x)
        if (h[i]) atomicAdd(&counts[i], h[i]);
}

size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Particle slots per CTA (ppc <= max_ppc) and warps per (slot, lag group)
// (parts): the most warps per CTA (at most 32), the larger ppc among equals.
// With 55 lags (two groups) and room for five slots this gives 4 slots x 4
// parts, 32 warps: 8.58e11 lag-pairs/s against 8.28e11 for 5 x 3 (30 warps).
constexpr int kMaxParts = 8;
void dmumu_shape(int max_ppc, int groups, int& ppc, int& parts)
{
    int best = 0;
    ppc = 1;
    parts = 1;
    for (int c = 1; c <= std::max(1, max_ppc) && c * groups <= 32; ++c) {
        const int pt = std::max(1, std::min(kMaxParts, 32 / (c * groups)));
        if (c * groups * pt >= best) {
            best = c * groups * pt;
            ppc = c;
            parts = pt;
        }
    }
}

}  // namespace

// ------------------------------------------------------------------ host side
namespace {

// D_mumu over the series that `src` yields (a.mu, a.sp, a.ss are not used here)
template <class Src>
int run_dmumu_src(pt_ctx* ctx, const DmumuArgs& a, const Src& src, cudaStream_t s)
{
    using MuT = typename Src::T;
    if (a.n <= 0 || a.n_lags <= 0) return PT_OK;
    if (a.n_bins < 1 || a.n_bins > 4096) return fail(PT_ERR_ARG, "n_bins must be in [1, 4096]");
    if (a.nsave < 1) return fail(PT_ERR_ARG, "nsave must be positive");
    int dev = ctx->device;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t budget = (size_t)std::min(max_smem, 200 * 1024);
    const bool small_idx = a.nsave <= 65535;
    const size_t idx_bytes = small_idx ? 2 : 4;
    const size_t edge_bytes = align16(sizeof(double) * (size_t)(a.n_bins + 1));
    // lags per launch: multiple of 32 with the accumulators taking <= ~half the budget
    int nl_cap = (int)std::max<size_t>(32, ((budget / 2) / ((size_t)a.n_bins * 24)) / 32 * 32);
    nl_cap = std::min(nl_cap, 32 * 8);
    const size_t slot_bytes = dmumu_slot_bytes(a.nsave, sizeof(MuT), idx_bytes, a.n_bins, nl_cap);
    const int lag_batches = (a.n_lags + nl_cap - 1) / nl_cap;
    for (int lb = 0; lb < lag_batches; ++lb) {
        const int lag0 = lb * nl_cap;
        const int nl = std::min(nl_cap, a.n_lags - lag0);
        const int groups = (nl + kWarp - 1) / kWarp;
        const size_t acc_bytes = (size_t)nl * a.n_bins * 24;
        size_t fixed = edge_bytes + std::max(acc_bytes, sizeof(WelfordPart) * 1024);
        bool smem_slots = fixed + slot_bytes <= budget;
        // more warps share each staged series: its start list is split over `parts` warps
        int ppc, parts;
        dmumu_shape(smem_slots ? (int)std::min<size_t>((budget - fixed) / slot_bytes, 32) : 8, groups, ppc, parts);
        const int threads = ppc * groups * parts * kWarp;
        size_t smem = fixed + (smem_slots ? (size_t)ppc * slot_bytes : 0);
        const int64_t tiles = (a.n + ppc - 1) / ppc;
        int per_sm = 1;
        void* kfn = small_idx ? (smem_slots ? (void*)dmumu_kernel<uint16_t, true, Src>
                                           : (void*)dmumu_kernel<uint16_t, false, Src>)
                              : (smem_slots ? (void*)dmumu_kernel<uint32_t, true, Src>
                                            : (void*)dmumu_kernel<uint32_t, false, Src>);
        PT_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem);
        per_sm = std::max(1, per_sm);
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)ctx->num_sms * per_sm));
        // scratch: per-CTA partials (+ global staging slots when needed)
        const size_t part_acc = (size_t)grid * nl * a.n_bins;
        const size_t bytes = align16(part_acc * 8) * 3 + align16(sizeof(WelfordPart) * (size_t)grid * nl) +
                             (smem_slots ? 0 : (size_t)grid * ppc * slot_bytes);
        void* scratch = nullptr;
        int rc = scratch_get(ctx, 0, bytes, &scratch);
        if (rc) return rc;
        char* base = (char*)scratch;
        DmumuLaunch L;
        L.n = a.n; L.nsave = a.nsave;
        L.start_cap = a.injection ? 1 : a.nsave;
        L.lags = a.lags + lag0; L.nl = nl; L.edges = a.edges; L.n_bins = a.n_bins; L.bin_abs = a.bin_abs;
        L.ppc = ppc; L.groups = groups; L.parts = parts; L.slot_bytes = slot_bytes;
        L.part_cnt = (unsigned long long*)base;
        L.part_sd = (double*)(base + align16(part_acc * 8));
        L.part_sd2 = (double*)(base + 2 * align16(part_acc * 8));
        L.part_w = (WelfordPart*)(base + 3 * align16(part_acc * 8));
        L.gslots = smem_slots ? nullptr : (char*)L.part_w + align16(sizeof(WelfordPart) * (size_t)grid * nl);
        if (small_idx) {
            if (smem_slots) dmumu_kernel<uint16_t, true, Src><<<grid, threads, smem, s>>>(L, src);
            else dmumu_kernel<uint16_t, false, Src><<<grid, threads, smem, s>>>(L, src);
        } else {
            if (smem_slots) dmumu_kernel<uint32_t, true, Src><<<grid, threads, smem, s>>>(L, src);
            else dmumu_kernel<uint32_t, false, Src><<<grid, threads, smem, s>>>(L, src);
        }
        PT_CHECK_LAUNCH("dmumu_kernel");
        const int fin_threads = 256;
        const int fin_blocks = (int)((std::max(nl * a.n_bins, nl) + fin_threads - 1) / fin_threads);
        dmumu_finalize_kernel<<<fin_blocks, fin_threads, 0, s>>>(L.part_cnt, L.part_sd, L.part_sd2, L.part_w, grid, nl,
                                                                 a.n_bins, lag0, a.n_lags, a.counts, a.sum_d,
                                                                 a.sum_d2, a.w_count, a.w_mean, a.w_m2, a.pair_ss,
                                                                 a.pair_n);
        PT_CHECK_LAUNCH("dmumu_finalize_kernel");
    }
    return PT_OK;
}

}  // namespace

int run_dmumu(pt_ctx* ctx, const DmumuArgs& a, cudaStream_t s)
{
    return run_dmumu_src(ctx, a, CacheSource{a.mu, a.sp, a.ss}, s);
}

namespace {

// (Bx, By, Bz) column-major arrays -> one record per node
template <typename R>
__global__ void interleave_b_kernel(const R* __restrict__ bx, const R* __restrict__ by, const R* __restrict__ bz,
                                    int64_t nodes, exact::Vec4<R>* __restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = exact::Vec4<R>{bx[i], by[i], bz[i], R(0)};
}

// (Bx, By, Bz) column-major arrays -> one 8-corner record per cell, indexed
// by the cell's base node (nodes on the last x, y or z plane are no base and
// their records are left unwritten: a sample never reads them).  Thread per
// record: the corner reads of neighbouring threads coalesce, and so do the
// record writes.
template <typename R>
__global__ void cell_b_kernel(const R* __restrict__ bx, const R* __restrict__ by, const R* __restrict__ bz, int64_t nx,
                              int64_t ny, int64_t nz, exact::CellB<R>* __restrict__ out)
{
    const int64_t nodes = nx * ny * nz, sy = nx, sz = nx * ny;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ix = i % nx, iy = (i / nx) % ny, iz = i / sz;
        if (ix >= nx - 1 || iy >= ny - 1 || iz >= nz - 1) continue;
        const int64_t off[8] = {0, 1, sy, 1 + sy, sz, 1 + sz, sy + sz, 1 + sy + sz};
        exact::CellB<R> r;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            r.v[3 * q] = bx[i + off[q]];
            r.v[3 * q + 1] = by[i + off[q]];
            r.v[3 * q + 2] = bz[i + off[q]];
        }
        out[i] = r;
    }
}

// mu of particles [p0, p0 + m) at every save, written [s][p - p0] (particle
// fastest, like the device mu cache); one thread per (particle, save),
// particles fastest so that the phase-space reads coalesce.  B comes from
// cell records (CELLS) or node records.
template <typename R, bool CELLS>
__global__ void __launch_bounds__(256) phase_space_mu_kernel(const R* __restrict__ pos, const R* __restrict__ mom,
                                                             int64_t row, int64_t comp, int64_t p0, int64_t m,
                                                             int64_t nsave, const void* __restrict__ Bsrc, pt_grid g,
                                                             R* __restrict__ mu)
{
    const int64_t total = m * nsave;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = t % m, s = t / m;
        const R* P = pos + s * row + p0 + q;
        const R* M = mom + s * row + p0 + q;
        if constexpr (CELLS)
            mu[s * m + q] = exact::phase_space_mu_cell<R>(P[0], P[comp], P[2 * comp], M[0], M[comp], M[2 * comp],
                                                          (const exact::CellB<R>*)Bsrc, g);
        else
            mu[s * m + q] = exact::phase_space_mu4<R>(P[0], P[comp], P[2 * comp], M[0], M[comp], M[2 * comp],
                                                      (const exact::Vec4<R>*)Bsrc, g);
    }
}

template <typename R>
int run_dmumu_phase_space_t(pt_ctx* ctx, const DmumuArgs& a, const R* pos, const R* mom, int64_t row, int64_t comp,
                            const void* const bfield[3], const pt_grid& g, cudaStream_t s)
{
    using V4 = exact::Vec4<R>;
    using CB = exact::CellB<R>;
    const int64_t nodes = g.nx * g.ny * g.nz;
    // mu chunks of at most 1 GiB
    const int64_t per = std::max<int64_t>(1, ((int64_t)1 << 30) / ((int64_t)sizeof(R) * a.nsave));
    const int64_t m_max = std::min<int64_t>(a.n, per);
    const size_t mu_bytes = sizeof(R) * (size_t)m_max * (size_t)a.nsave;
    // B as cell records when they take at most half of the free device
    // memory: a sample then reads one 96-byte (FP32) record instead of 8
    // node records from 4 grid rows, ~4x fewer DRAM bytes on the random
    // gathers of particles in id order; otherwise as node records
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = 0;
    }
    const size_t cell_bytes = align16(sizeof(CB) * (size_t)nodes);
    bool cells = cell_bytes + mu_bytes <= free_b / 2;
    // PTB200_PHASE_SPACE_B = "nodes" or "cells" overrides the choice (same results)
    if (const char* e = std::getenv("PTB200_PHASE_SPACE_B")) {
        if (!std::strcmp(e, "nodes")) cells = false;
        else if (!std::strcmp(e, "cells")) cells = true;
    }
    const size_t b_bytes = cells ? cell_bytes : align16(sizeof(V4) * (size_t)nodes);
    void* scratch = nullptr;
    int rc = scratch_get(ctx, 4, b_bytes + mu_bytes, &scratch);
    if (rc) return rc;
    R* mu = (R*)((char*)scratch + b_bytes);
    const int gb = (int)std::min<int64_t>((nodes + 255) / 256, (int64_t)ctx->num_sms * 16);
    if (cells) {
        cell_b_kernel<R><<<gb, 256, 0, s>>>((const R*)bfield[0], (const R*)bfield[1], (const R*)bfield[2], g.nx, g.ny,
                                            g.nz, (CB*)scratch);
        PT_CHECK_LAUNCH("cell_b_kernel");
    } else {
        interleave_b_kernel<R><<<gb, 256, 0, s>>>((const R*)bfield[0], (const R*)bfield[1], (const R*)bfield[2], nodes,
                                                  (V4*)scratch);
        PT_CHECK_LAUNCH("interleave_b_kernel");
    }
    for (int64_t p0 = 0; p0 < a.n; p0 += m_max) {
        const int64_t m = std::min(m_max, a.n - p0);
        const int64_t total = m * a.nsave;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 32);
        if (cells)
            phase_space_mu_kernel<R, true><<<blocks, 256, 0, s>>>(pos, mom, row, comp, p0, m, a.nsave, scratch, g, mu);
        else
            phase_space_mu_kernel<R, false><<<blocks, 256, 0, s>>>(pos, mom, row, comp, p0, m, a.nsave, scratch, g, mu);
        PT_CHECK_LAUNCH("phase_space_mu_kernel");
        DmumuArgs c = a;
        c.n = m;
        rc = run_dmumu_src(ctx, c, CacheSourceT<R>{mu, 1, m}, s);
        if (rc) return rc;
    }
    return PT_OK;
}

}  // namespace

int run_dmumu_phase_space(pt_ctx* ctx, const DmumuArgs& a, const void* pos, const void* mom, int64_t row,
                          int64_t comp, const void* const bfield[3], const pt_grid& g, int f64, cudaStream_t s)
{
    if (a.n <= 0 || a.n_lags <= 0) return PT_OK;
    if (f64) return run_dmumu_phase_space_t<double>(ctx, a, (const double*)pos, (const double*)mom, row, comp, bfield,
                                                    g, s);
    return run_dmumu_phase_space_t<float>(ctx, a, (const float*)pos, (const float*)mom, row, comp, bfield, g, s);
}

int run_dpp(pt_ctx* ctx, const DppArgs& a, cudaStream_t s)
{
    if (a.chunk <= 0 || a.n_lags <= 0) return PT_OK;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    const size_t budget = (size_t)std::min(max_smem, 200 * 1024);
    if (a.nsave >= INT32_MAX) return fail(PT_ERR_ARG, "nsave must be below 2^31");
    const size_t slot_bytes = align16(sizeof(double) * (size_t)(a.nsave + 1));  // + NaN pad
    const int nl_cap = 32 * 8;
    for (int lag0 = 0; lag0 < a.n_lags; lag0 += nl_cap) {
        const int nl = std::min(nl_cap, a.n_lags - lag0);
        // particle slots per CTA (series on chip when they fit) and warps per
        // slot (each takes ceil(nl / wps) lags, two at a time)
        const size_t acc_per_slot = sizeof(DppPart) * (size_t)nl;
        bool smem_slots = align16(acc_per_slot) + slot_bytes <= budget;
        // the most warps per CTA (at most 32), the larger ppc among equals:
        // at 55 lags and room for five series, 4 slots x 8 warps measured
        // 1.45e12 lag-pairs/s against 1.32e12 for 5 x 6
        const int max_ppc = smem_slots ? (int)std::min<size_t>(budget / (slot_bytes + acc_per_slot), 8) : 4;
        const int lag_sets = (nl + kDppLags - 1) / kDppLags;
        int ppc = 1, wps = 1, best = 0;
        for (int c = 1; c <= std::max(1, max_ppc); ++c) {
            const int w = std::max(1, std::min(32 / c, lag_sets));
            if (c * w >= best) {
                best = c * w;
                ppc = c;
                wps = w;
            }
        }
        const int threads = ppc * wps * kWarp;
        const size_t smem = align16(acc_per_slot * ppc) + (smem_slots ? (size_t)ppc * slot_bytes : 0);
        const int64_t tiles = (a.chunk + ppc - 1) / ppc;
        void* kfn = smem_slots ? (void*)dpp_kernel<true> : (void*)dpp_kernel<false>;
        PT_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem);
        per_sm = std::max(1, per_sm);
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)ctx->num_sms * per_sm));
        const size_t bytes = align16(sizeof(DppPart) * (size_t)grid * nl) +
                             (smem_slots ? 0 : (size_t)grid * ppc * slot_bytes);
        void* scratch = nullptr;
        int rc = scratch_get(ctx, 1, bytes, &scratch);
        if (rc) return rc;
        DppLaunch L;
        L.mom = a.mom; L.chunk = a.chunk; L.nsave = a.nsave; L.lags = a.lags + lag0; L.nl = nl; L.p0 = a.p0;
        L.ppc = ppc; L.wps = wps; L.slot_bytes = slot_bytes;
        L.part = (DppPart*)scratch;
        L.gslots = smem_slots ? nullptr : (char*)scratch + align16(sizeof(DppPart) * (size_t)grid * nl);
        if (smem_slots) dpp_kernel<true><<<grid, threads, smem, s>>>(L);
        else dpp_kernel<false><<<grid, threads, smem, s>>>(L);
        PT_CHECK_LAUNCH("dpp_kernel");
        dpp_finalize_kernel<<<(nl + 255) / 256, 256, 0, s>>>(L.part, grid, nl, lag0, a.p0, a.counts, a.sdp, a.sdp2,
                                                             a.sdn, a.sdn2);
        PT_CHECK_LAUNCH("dpp_finalize_kernel");
    }
    return PT_OK;
}

int launch_energy_snapshots(const float* mom, int64_t chunk, int64_t nsave, const int64_t* snaps, int n_snap,
                            int64_t offset, double* out, cudaStream_t s)
{
    const int64_t total = chunk * n_snap;
    if (total <= 0) return PT_OK;
    energy_snap_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(mom, chunk, nsave, snaps, n_snap, offset, out);
    PT_CHECK_LAUNCH("energy_snap_kernel");
    return PT_OK;
}

int launch_energy_histogram(const float* mom, int64_t chunk, int64_t nsave, const int64_t* snaps, int n_snap,
                            double e_min, double e_max, int n_hist, int64_t* counts, cudaStream_t s)
{
    const int64_t total = chunk * n_snap;
    if (total <= 0) return PT_OK;
    const size_t smem = sizeof(unsigned long long) * (size_t)n_snap * n_hist;
    if (smem > 160 * 1024) return fail(PT_ERR_ARG, "n_snap * n_hist too large for the on-chip histogram");
    if (smem > 48 * 1024)
        PT_CUDA(cudaFuncSetAttribute(energy_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const double log_emin = log(e_min);
    const double inv_dlog = (double)n_hist / (log(e_max) - log_emin);
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 4);
    energy_hist_kernel<<<blocks, 256, smem, s>>>(mom, chunk, nsave, snaps, n_snap, log_emin, inv_dlog, n_hist,
                                                 (unsigned long long*)counts);
    PT_CHECK_LAUNCH("energy_hist_kernel");
    return PT_OK;
}

}  // namespace pt

// ---------------------------------------------------------------------------
// D_mumu accumulation that allocates nothing.
//
// Some callers cannot let a library allocate device memory: a host that owns
// all device memory through its own pool (the Julia host's CUDA.jl pool, or
// the campaign server's HBM-budget admission) has no way to account for a
// cudaMalloc made behind its back, and cudaFree synchronises the whole
// device, stalling every other stream of a busy GPU.  For them the per-CTA
// partials of the D_mumu kernel live in a fixed, file-scope device array of
// kDmumuNoAllocBytes (16 MiB) that every GPU which loads the library holds
// until the process exits.  The array's device address is looked up once per
// device with cudaGetSymbolAddress (host code cannot use the symbol itself:
// on the host it names a stand-in, not device memory).
// ---------------------------------------------------------------------------
#include <mutex>

static constexpr size_t kDmumuNoAllocBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_dmumu_noalloc_scratch[kDmumuNoAllocBytes];

namespace pt {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the fixed scratch on `device` (set up on first use).
int noalloc_scratch(int device, void** out)
{
    if (device < 0 || device >= kMaxDevices) return fail(PT_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        int prev = 0;
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
        e = cudaSetDevice(device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_dmumu_noalloc_scratch);
        cudaError_t e2 = cudaSetDevice(prev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_dmumu_noalloc_scratch)");
        if (e2 != cudaSuccess) return cuda_fail(e2, "cudaSetDevice");
        g_noalloc_ptr[device] = p;
    }
    *out = g_noalloc_ptr[device];
    return PT_OK;
}

int run_dmumu_noalloc(pt_ctx* ctx, const DmumuArgs& a, cudaStream_t s)
{
    if (a.n <= 0 || a.n_lags <= 0) return PT_OK;
    if (a.n_bins < 1 || a.n_bins > 4096) return fail(PT_ERR_ARG, "n_bins must be in [1, 4096]");
    if (a.nsave < 1) return fail(PT_ERR_ARG, "nsave must be positive");
    void* scratch = nullptr;
    int rc = noalloc_scratch(ctx->device, &scratch);
    if (rc) return rc;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    const size_t budget = (size_t)std::min(max_smem, 200 * 1024);
    const bool small_idx = a.nsave <= 65535;
    const size_t idx_bytes = small_idx ? 2 : 4;
    const size_t edge_bytes = align16(sizeof(double) * (size_t)(a.n_bins + 1));
    int nl_cap = (int)std::max<size_t>(32, ((budget / 2) / ((size_t)a.n_bins * 24)) / 32 * 32);
    nl_cap = std::min(nl_cap, 32 * 8);
    const size_t slot_bytes = dmumu_slot_bytes(a.nsave, sizeof(float), idx_bytes, a.n_bins, nl_cap);
    const CacheSource src{a.mu, a.sp, a.ss};
    for (int lag0 = 0; lag0 < a.n_lags; lag0 += nl_cap) {
        const int nl = std::min(nl_cap, a.n_lags - lag0);
        const int groups = (nl + kWarp - 1) / kWarp;
        const size_t acc_bytes = (size_t)nl * a.n_bins * 24;
        const size_t fixed = edge_bytes + std::max(acc_bytes, sizeof(WelfordPart) * 1024);
        if (fixed + slot_bytes > budget)
            return fail(PT_ERR_ARG, "pt_dmumu_accumulate_device_noalloc: nsave = " + std::to_string(a.nsave) +
                                        " is too long for on-chip staging with " + std::to_string(a.n_bins) +
                                        " bins; use pt_dmumu_accumulate_device");
        int ppc, parts;
        dmumu_shape((int)std::min<size_t>((budget - fixed) / slot_bytes, 32), groups, ppc, parts);
        const int threads = ppc * groups * parts * kWarp;
        const size_t smem = fixed + (size_t)ppc * slot_bytes;
        // per-CTA partials: counts, sum, sum^2 per (lag, bin) and a Welford triple per lag
        const size_t per_cta = (size_t)nl * a.n_bins * 24 + sizeof(WelfordPart) * (size_t)nl + 64;
        const int64_t cap_grid = (int64_t)((kDmumuNoAllocBytes - 1024) / per_cta);
        if (cap_grid < 1)
            return fail(PT_ERR_ARG, "pt_dmumu_accumulate_device_noalloc: n_lags x n_bins too large for the " +
                                        std::to_string(kDmumuNoAllocBytes >> 20) + " MiB fixed scratch");
        void* kfn = small_idx ? (void*)dmumu_kernel<uint16_t, true, CacheSource>
                              : (void*)dmumu_kernel<uint32_t, true, CacheSource>;
        PT_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem);
        per_sm = std::max(1, per_sm);
        const int64_t tiles = (a.n + ppc - 1) / ppc;
        const int grid = (int)std::max<int64_t>(
            1, std::min<int64_t>(std::min<int64_t>(tiles, (int64_t)ctx->num_sms * per_sm), cap_grid));
        const size_t part_acc = (size_t)grid * nl * a.n_bins;
        char* base = (char*)scratch;
        DmumuLaunch L;
        L.n = a.n; L.nsave = a.nsave;
        L.start_cap = a.injection ? 1 : a.nsave;
        L.lags = a.lags + lag0; L.nl = nl; L.edges = a.edges; L.n_bins = a.n_bins; L.bin_abs = a.bin_abs;
        L.ppc = ppc; L.groups = groups; L.parts = parts; L.slot_bytes = slot_bytes;
        L.part_cnt = (unsigned long long*)base;
        L.part_sd = (double*)(base + align16(part_acc * 8));
        L.part_sd2 = (double*)(base + 2 * align16(part_acc * 8));
        L.part_w = (WelfordPart*)(base + 3 * align16(part_acc * 8));
        L.gslots = nullptr;
        if (3 * align16(part_acc * 8) + sizeof(WelfordPart) * (size_t)grid * nl > kDmumuNoAllocBytes)
            return fail(PT_ERR_ARG, "internal: no-alloc scratch overflow");
        if (small_idx) dmumu_kernel<uint16_t, true, CacheSource><<<grid, threads, smem, s>>>(L, src);
        else dmumu_kernel<uint32_t, true, CacheSource><<<grid, threads, smem, s>>>(L, src);
        PT_CHECK_LAUNCH("dmumu_kernel (no-alloc)");
        const int fin_blocks = (int)((std::max(nl * a.n_bins, nl) + 255) / 256);
        dmumu_finalize_kernel<<<fin_blocks, 256, 0, s>>>(L.part_cnt, L.part_sd, L.part_sd2, L.part_w, grid, nl,
                                                         a.n_bins, lag0, a.n_lags, a.counts, a.sum_d, a.sum_d2,
                                                         a.w_count, a.w_mean, a.w_m2, a.pair_ss, a.pair_n);
        PT_CHECK_LAUNCH("dmumu_finalize_kernel (no-alloc)");
    }
    return PT_OK;
}

}  // namespace
}  // namespace pt

extern "C" int pt_dmumu_accumulate_device_noalloc(pt_ctx* ctx, const float* d_mu, int64_t n, int64_t nsave, int64_t sp,
                                                  int64_t ss, const int64_t* d_lags, int n_lags, const double* d_edges,
                                                  int n_bins, int start_mode, int bin_abs, int64_t* d_counts,
                                                  double* d_sum_d, double* d_sum_d2, int64_t* d_w_count,
                                                  double* d_w_mean, double* d_w_m2, double* d_pair_ss,
                                                  int64_t* d_pair_n)
{
    using namespace pt;
    if (!ctx) return fail(PT_ERR_ARG, "ctx is null");
    if (n < 0 || nsave < 1 || n_lags < 0 || n_bins < 1) return fail(PT_ERR_ARG, "bad sizes");
    if (start_mode != PT_START_SLIDING && start_mode != PT_START_INJECTION) return fail(PT_ERR_ARG, "start_mode");
    if (n == 0 || n_lags == 0) return PT_OK;
    if (!(d_mu && d_lags && d_edges && d_counts && d_sum_d && d_sum_d2 && d_w_count && d_w_mean && d_w_m2 &&
          d_pair_ss && d_pair_n))
        return fail(PT_ERR_ARG, "null pointer");
    PT_DEVICE_SCOPE(ctx->device);
    DmumuArgs a{d_mu, n, nsave, sp, ss, d_lags, n_lags, d_edges, n_bins, start_mode == PT_START_INJECTION, bin_abs != 0,
                d_counts, d_sum_d, d_sum_d2, d_w_count, d_w_mean, d_w_m2, d_pair_ss, d_pair_n};
    return run_dmumu_noalloc(ctx, a, ctx->stream);
}
