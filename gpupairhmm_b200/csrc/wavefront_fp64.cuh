// FP64 pass: the same wavefront in double precision for the pairs the FP32
// pass flagged (scaled FP32 sum below the underflow threshold, or an alpha
// too close to zero for the FP32 kernel's division).  Two tiers:
//
// Scaled tier (EXT = false): plain doubles under one fixed power-of-two scale.
// The D boundary enters at 2^kScaledExp times the reference's FLT_MAX/16 scale
// (values start near 2^960, leaving 2^63 of headroom for the rescaled
// variables, which exceed the true values by at most 1/q and 1/s < 2^45).  A
// cell's share of the result is at most its value, and each of the five
// roundings of a cell moves a true value by at most 2^-1075 in the subnormal
// range, so a sum S >= L*H*2^-1030 is exact to 5*2^-45 relative; that covers
// pairs down to about 10^-599 * L*H.  Pairs below it (or non-finite) go on to
// the extended tier's list; a multi-tile pair goes there as soon as the mass on
// a tile's border column (an upper bound of its final sum) is below half the
// threshold, skipping its remaining tiles.  With fuse (multi-tile class, small
// batches) the pair is not listed: the same warp runs its extended form next.  No exponent bookkeeping: a step is
// the R cells, the hand-off shuffles and the table loads.
//
// Extended tier (EXT = true): an unrelated read far longer than its haplotype
// lies thousands of decades below 1, beyond a pre-scaled double.  Every lane
// therefore stores its values as
// true * 2^e  with its own integer exponent e.  A lane centres its exponent
// on the first non-zero values it receives (its neighbour may not have
// renormalised yet), every 16 steps it renormalises its registers by an exact
// power of two, and every value handed to the next lane travels with the
// sender's exponent; the receiver multiplies it by 2^(e_recv - e_send).  The
// result lane keeps its accumulator in its own scale and renormalises it with
// its registers, so the result is
//     log10(acc) - e*log10(2) - log10(beta*FLT_MAX/16).
// Values more than 2^1022 below the largest value of their lane are dropped;
// their contribution to the result is below that factor too.
//
// The recurrence runs in the rescaled variables of the FP32 kernel: I and D
// divided by the weight of the term that feeds them (q_c = beta*delta_c, or
// beta from the read end on; s_c = beta*sigma_c), and the diagonal sum
// X = I + D(j-1) divided by q_c, with q_{c-1} folded into the lambda table
// and alpha_c/q_{c-1} kept per position:
//     D^(j,c) = eps*D^(j-1,c) + M(j-1,c)
//     I^(j,c) = e_c*I^(j,c-1) + M(j-1,c-1),        e_c = eps_c*q_{c-1}/q_c
//     X^(j,c) = (s_c/q_c)*D^(j-1,c) + I^(j,c)
//     M(j,c)  = lambda*q_{c-1} * ((alpha_c/q_{c-1})*M(j-1,c-1) + X^(j,c-1))
// Five double operations per cell (four DFMA, one DMUL).  Nothing divides by
// alpha, so pairs with alpha near or at zero are exact here.  The read-end
// carry is that of the FP32 kernel (eps = 1 and scale beta from the read end).
//
// Work split as in the FP32 kernel: groups of G lanes, R doubles per lane,
// T = G*R read positions per tile; reads longer than T (MT, G = 32 only) run
// tile after tile with the last lane's (M, Dt, It, exponents) per haplotype
// row going through a global border buffer, staged through a 32-entry shared
// ring for lane 0 of the next tile.  One buffer serves every tile boundary of
// a pair: tile i+1 reads a row (ring prefetch, up to 64 rows ahead) before its
// own last lane overwrites it 31 steps later, in the same warp.
#pragma once

#include <climits>
#include <type_traits>

#include "device_common.cuh"

namespace phmm {

// Border row between read tiles: M of row s, X^ and I^ of row s + 1.  The
// extended tier carries the exponents too; the scaled tier needs none.
struct Border64 {
    double m, x, i;
    int e;   // exponent of m (row s)
    int ei;  // exponent of x and i (row s + 1)
};
static_assert(sizeof(Border64) == 32, "Border64 is 32 bytes");
struct Border64S {
    double m, x, i;
};
static_assert(sizeof(Border64S) == 24, "Border64S is 24 bytes");

template <bool EXT>
__device__ __forceinline__ void border_set_m(Border64& b, double m, int e) { b.m = m; b.e = e; }
template <bool EXT>
__device__ __forceinline__ void border_set_m(Border64S& b, double m, int) { b.m = m; }
template <bool EXT>
__device__ __forceinline__ void border_set_xi(Border64& b, double x, double i, int e) { b.x = x; b.i = i; b.ei = e; }
template <bool EXT>
__device__ __forceinline__ void border_set_xi(Border64S& b, double x, double i, int) { b.x = x; b.i = i; }
__device__ __forceinline__ int border_e(const Border64& b) { return b.e; }
__device__ __forceinline__ int border_e(const Border64S&) { return 0; }
__device__ __forceinline__ int border_ei(const Border64& b) { return b.ei; }
__device__ __forceinline__ int border_ei(const Border64S&) { return 0; }

// 2^k as a double for k clamped to the normal range (exact power of two)
__device__ __forceinline__ double pow2i(int k) {
    k = k < -1022 ? -1022 : (k > 1023 ? 1023 : k);
    return __longlong_as_double((long long)(k + 1023) << 52);
}

// Scaled tier: the D boundary's power-of-two factor over the reference's scale,
// and the smallest sum it keeps (relative error of the subnormal roundings
// below 5*2^-45 above it).
constexpr int kScaledExp = 836;
__host__ __device__ __forceinline__ double scaled_tier_threshold(int L, int H) {
    return (double)L * (double)H * 0x1p-1030;
}

template <int G, int R, bool MT, bool GCP = false, bool EXT = true>
struct Fp64Wavefront {
    static_assert(R % 2 == 0, "R must be even");
    static_assert(!MT || G == 32, "multi-tile FP64 runs one pair per warp");
    static constexpr int NG = 32 / G;
    static constexpr int T = G * R;
    static constexpr int G_ = G, R_ = R;
    static constexpr bool kMT = MT, kGCP = GCP, kEXT = EXT;
    static constexpr int Q = R / 2;                   // double2 per thread per table row
    static constexpr int kTableDouble2 = 5 * Q * 32;  // per warp
    static constexpr int kRing = 32;
    // border rows sit kRowPad entries into the warp's buffer: the last lane writes row
    // k - (G - 1) at step k from k = 0 on, without bounds branches (rows before 0 and
    // after the haplotype's last fall in the padding; the buffer has at least
    // max H + 72 rows, and the last write of a tile is row H + 4)
    static constexpr int kRowPad = G;
    using Border = typename std::conditional<EXT, Border64, Border64S>::type;
    // largest scale difference a hand-off converts: stored values stay within
    // about 2^(64 + 13*16) of 1 between renormalisations, so 2^640 more keeps
    // every converted value below 2^1023
    static constexpr int kMaxShift = 640;
    // resident 64-thread CTAs per SM asked of the register allocator: the
    // 10-position tile allocates about 200 registers (2 warps per scheduler),
    // capped at 168 it keeps 3; the 8-position single tiles allocate about 158,
    // capped at 128 they keep 4
    static constexpr int kMinCtas = R == 10 ? 6 : (R == 8 && !MT) ? 8 : 1;

    // tasks: the warp's ntask (<= NG) items.  wtab: this warp's lambda table;
    // ring: kRing shared entries (MT); scratch: this warp's rows border entries.
    // ext: the extended tier's lists (scaled tier only).
    // fuse (multi-tile scaled tier only): a pair that needs the extended tier is not
    // appended to its list; run returns true and the caller runs the extended form
    __device__ static bool run(const DevView& v, const Task* tasks, int ntask, const float* ph, double2* wtab,
                               Border* ring, Border* scratch, int64_t rows, const ExtList& ext, bool fuse) {
        const int lane = threadIdx.x & 31;
        const int grp = lane / G;
        const int t = lane - grp * G;
        const bool active = grp < ntask;
        const Task task = tasks[active ? grp : 0];
        const int L = v.read_len[task.read];
        const int H = v.hap_len[task.hap];
        const bool valid = active && L >= 1 && H >= 1;
        const int Lc = L >= 1 ? L : 1;
        const int Hc = H >= 1 ? H : 1;
        const int ntiles = MT ? (Lc + T - 1) / T : 1;  // MT: one group, warp-uniform
        const uint32_t* rpack = v.read_pack + v.read_start[task.read];
        const uint32_t* hw = reinterpret_cast<const uint32_t*>(v.hap_code + v.hap_start[task.hap]);
        // gcp mode: the read's own eps and beta (gpuworker.cuh:1048-1049), as the
        // FP32 kernel forms them; beta = 0 (gcp quality 0) has no rescaled form
        const float eps_f = GCP ? ph[v.read_gcp[task.read]] : kEps;
        const double beta = GCP ? (double)(float)(1.0 - (double)eps_f) : (double)kBeta;
        const double epsd = (double)eps_f;
        const double Dbound = beta * (double)(kScale / (float)Hc) * (EXT ? 1.0 : 0x1p836);
        static_assert(kScaledExp == 836, "scale literal");

        double acc = 0.0;
        int e = EXT ? 0 : kScaledExp;
        int eacc = e;  // exponent of acc: the lane's e up to the pair's last step, then frozen
        int rlane = -1;

        for (int tile = 0; tile < ntiles; ++tile) {
            const bool last = tile == ntiles - 1;
            const int p0 = tile * T + t * R;
            // I scale of the position before this lane's first (1 at the read's column -1)
            double qp = 1.0;
            if (p0 > 0) {
                qp = beta;
                if (p0 - 1 < L) qp = beta * (double)ph[(__ldg(rpack + p0 - 1) >> 16) & 0x7fu];
            }
            double aq[R], ee[R], rr[R], M[R], D[R];
            // one division per position: 1/q of the previous position is carried
            double iqp = 1.0 / qp;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                double lam[5][2];
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int r = 2 * q + s;
                    const int c = p0 + r;
                    const bool in = c < L;
                    const uint32_t w = in ? __ldg(rpack + c) : 0u;
                    const uint32_t x = w & 0xffu;
                    const float p = ph[(w >> 8) & 0x7fu];
                    const float d = ph[(w >> 16) & 0x7fu];
                    const float sg = ph[(w >> 24) & 0x7fu];
                    const double lm = (double)(1.0f - p) * qp;
                    const double lx = (double)(p / 3.0f) * qp;
#pragma unroll
                    for (int h = 0; h < 5; ++h)
                        lam[h][s] = in ? ((x == 4u || h == 4 || x == (uint32_t)h) ? lm : lx) : 0.0;
                    const double qc = in ? beta * (double)d : beta;
                    const double iqc = 1.0 / qc;
                    aq[r] = (double)(1.0f - (d + sg)) * iqp;
                    ee[r] = ((in ? epsd : 1.0) * qp) * iqc;
                    rr[r] = in ? (beta * (double)sg) * iqc : 0.0;
                    qp = qc;
                    iqp = iqc;
                    M[r] = 0.0;
                    D[r] = 0.0;
                }
#pragma unroll
                for (int h = 0; h < 5; ++h) wtab[(h * Q + q) * 32 + lane] = make_double2(lam[h][0], lam[h][1]);
            }
            if constexpr (EXT) e = 0;
            int t_res = 0, r_res = 0;
            if (last) {
                const int rel = Lc - 1 - tile * T;
                t_res = rel / R;
                r_res = rel - t_res * R;
            }
            const int kg = last ? Hc + t_res : Hc + G - 1;
            const bool res_lane = valid && last && t == t_res;
            const bool addM = r_res == R - 1;
            // weight of the lane's last I^ in the result: beta in the carry, q when
            // the read ends on the lane's last position
            const double qres = addM ? qp : beta;
            if (res_lane) rlane = t;
            const int kmax = (int)__reduce_max_sync(kFullMask, (unsigned)(valid ? kg : 0));
            const int K = (kmax + 1 + 3) & ~3;

            // left-boundary inputs: M(j-1) with exponent eMul, I^(j) and X^(j) with eIul
            // (read column -1: X = D = Dbound)
            double Ml = 0.0, Mul = 0.0, Iul = 0.0, Xul = 0.0;
            int eMl = 0, eMul = 0, eIul = 0;
            if (t == 0 && tile == 0) Xul = Dbound;
            bool empty = !(t == 0 && tile == 0);
            const Border* ein = scratch;
            Border* eout = scratch;
            const bool writer = MT && valid && !last && t == G - 1;
            Border nb{};
            if (MT && tile > 0 && t + kRowPad < rows) nb = ein[t + kRowPad];
            int h = 4;

            // code words of this group's haplotype, clamped to its own extent
            const int wlast = ((Hc + 15) & ~15) / 4 - 1;
            uint32_t wcur = __ldg(hw);
            uint32_t wnext = __ldg(hw + 1);
            for (int k0 = 0; k0 < K; k0 += 4) {
                const uint32_t wpref = __ldg(hw + min_i((k0 >> 2) + 2, wlast));
                if (MT && tile > 0 && (k0 & (kRing - 1)) == 0) {
                    __syncwarp();
                    ring[t] = nb;
                    __syncwarp();
                    const int64_t idx = (int64_t)k0 + kRing + t;
                    if (idx + kRowPad < rows) nb = ein[idx + kRowPad];
                }
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int k = k0 + s;
                    int hn = __shfl_up_sync(kFullMask, h, 1, G);
                    if (t == 0) hn = (int)((wcur >> (8 * s)) & 0xffu);
                    h = hn;
                    // lanes fill during the first pass of the wavefront (k < G + 8)
                    if (EXT && k0 < G + 8 && empty && (Mul != 0.0 || Xul != 0.0 || Iul != 0.0)) {
                        // centre this lane's scale on the first values it receives
                        const double xi = fmax(fabs(Xul), fabs(Iul));
                        e = Mul != 0.0 ? eMul - ilogb(fabs(Mul)) : eIul - ilogb(xi);
                        empty = false;
                    }
                    const double2* trow = wtab + h * (Q * 32) + lane;
                    if (EXT && e - (eMul < eIul ? eMul : eIul) > kMaxShift) {  // rare: one compare per step
                        // a neighbour's values far above this lane's scale (a lane centred on
                        // the tiny first values of a long insertion path meets the large ones
                        // that follow): coarsen the scale first, by an exact power of two, so
                        // the conversion below cannot overflow; this lane's values that fall
                        // out of range are negligible next to the incoming ones
                        const int dM = Mul != 0.0 ? e - eMul : INT_MIN;
                        const int dI = (Xul != 0.0 || Iul != 0.0) ? e - eIul : INT_MIN;
                        const int over = (dM > dI ? dM : dI) - kMaxShift;
                        if (over > 0) {
                            const double f = over > 1022 ? 0.0 : pow2i(-over);
#pragma unroll
                            for (int r = 0; r < R; ++r) { M[r] *= f; D[r] *= f; }
                            if (k <= kg) acc *= f;
                            e -= over;
                        }
                    }
                    // border row for the next step's diagonal, loaded before this step's cells
                    // so the shared-memory latency overlaps them (every lane takes part in the
                    // broadcast load, lane 0 keeps it)
                    Border bk{};
                    if (MT && tile > 0) bk = ring[k & (kRing - 1)];
                    double Mdiag = Mul, Idiag = Iul, Xdiag = Xul;
                    if constexpr (EXT) {
                        const double fM = pow2i(e - eMul);
                        const double fI = pow2i(e - eIul);
                        Mdiag *= fM;
                        Idiag *= fI;
                        Xdiag *= fI;
                    }
#pragma unroll
                    for (int q = 0; q < Q; ++q) {
                        const double2 lam = trow[q * 32];
                        const double ls[2] = {lam.x, lam.y};
#pragma unroll
                        for (int u = 0; u < 2; ++u) {
                            const int r = 2 * q + u;
                            const double Mold = M[r];
                            const double Dold = D[r];
                            M[r] = ls[u] * fma(aq[r], Mdiag, Xdiag);
                            D[r] = fma(epsd, Dold, Mold);
                            const double In = fma(ee[r], Idiag, Mdiag);
                            Xdiag = fma(rr[r], Dold, In);
                            Mdiag = Mold;
                            Idiag = In;
                        }
                    }
                    if (res_lane && k <= kg) {
                        acc = fma(qres, Idiag, acc);
                        if (addM && k < kg) acc = fma(beta, M[R - 1], acc);
                    }
                    if (writer) {
                        // slot s + kRowPad holds M(s), and X^(s+1), I^(s+1); rows before the
                        // haplotype and past it land in the padding and are never read
                        const int j = k - (G - 1);
                        border_set_m<EXT>(eout[j + kRowPad], M[R - 1], e);
                        border_set_xi<EXT>(eout[j - 1 + kRowPad], Xdiag, Idiag, e);
                    }
                    // hand-off: values travel with the sender's exponent
                    Mul = Ml; eMul = eMl;
                    Ml = __shfl_up_sync(kFullMask, M[R - 1], 1, G);
                    Iul = __shfl_up_sync(kFullMask, Idiag, 1, G);
                    Xul = __shfl_up_sync(kFullMask, Xdiag, 1, G);
                    if constexpr (EXT) {
                        const int es = __shfl_up_sync(kFullMask, e, 1, G);
                        eMl = es;
                        eIul = es;
                    }
                    if (MT && tile > 0) {
                        // the border is indexed by row: it feeds the next step's diagonal
                        if (t == 0) {
                            const bool in = k < Hc;
                            Mul = in ? bk.m : 0.0; Xul = in ? bk.x : 0.0; Iul = in ? bk.i : 0.0;
                            eMul = in ? border_e(bk) : 0; eIul = in ? border_ei(bk) : 0;
                        }
                    } else if (t == 0) {
                        Ml = 0.0; Iul = 0.0; Xul = Dbound; eMl = 0; eIul = 0;
                    }
                    // renormalise every 16 steps (exact powers of two); a value moves by at
                    // most 2^13 per row, so lanes stay within 2^300 of their scale meanwhile
                    if (EXT && (k & 15) == 15) {
                        // the hand-off values count too: past the read end M is zero and
                        // only the carried I^ and X^ move
                        double mx = fmax(res_lane && k <= kg ? fabs(acc) : 0.0, fmax(fabs(Idiag), fabs(Xdiag)));
#pragma unroll
                        for (int r = 0; r < R; ++r) mx = fmax(mx, fmax(fabs(M[r]), fabs(D[r])));
                        if (mx > 0.0) {
                            const int fe = ilogb(mx);
                            if (fe > 64 || fe < -64) {
                                const int kk = -fe < -1022 ? -1022 : (-fe > 1023 ? 1023 : -fe);
                                const double f = pow2i(kk);
#pragma unroll
                                for (int r = 0; r < R; ++r) { M[r] *= f; D[r] *= f; }
                                if (k <= kg) acc *= f;
                                e += kk;
                            }
                        }
                    }
                    // a group whose pair has ended keeps stepping while another group of
                    // the warp runs on; its values then are not the pair's and must not
                    // rescale the finished sum
                    if (k <= kg) eacc = e;
                }
                wcur = wnext;
                wnext = wpref;
            }
            __syncwarp();
            if constexpr (MT && !EXT) {
                // early hand-off to the extended tier: every path to the result crosses
                // this tile's border column once and nothing on it exceeds 1, so the final
                // sum is at most the border's mass, sum over rows of M + q*X^ (= M + I + D);
                // below half the tier's threshold the sum would fail it at the end too
                if (!last && !(GCP && !(beta > 0.0))) {
                    const double qlast = __shfl_sync(kFullMask, qp, G - 1);
                    double mass = 0.0;
                    for (int j = t - 1; j < Hc; j += G) {
                        const Border b = eout[j + kRowPad];
                        mass += b.m + qlast * b.x;
                    }
#pragma unroll
                    for (int d = 16; d >= 1; d >>= 1) mass += __shfl_xor_sync(kFullMask, mass, d);
                    if (mass < 0.5 * scaled_tier_threshold(L, H)) {  // warp-uniform: one pair per warp
                        if (fuse) return valid;
                        if (valid && t == 0) {
                            const int cls = fp64_class(L);
                            const unsigned long long slot = atomicAdd(ext.count + cls, 1ull);
                            ext.base[ext.off[cls] + (long long)slot] = task;
                        }
                        return false;  // no score: the extended tier writes it
                    }
                }
            }
        }
        // scaled tier: a sum too small (or not finite) for the fixed scale goes on to
        // the extended tier, which overwrites the score
        const bool to_ext = !EXT && valid && t == rlane && !(acc >= scaled_tier_threshold(L, H) && acc <= DBL_MAX) &&
                            !(GCP && !(beta > 0.0));
        if (valid && t == rlane) {
            double res = -INFINITY;
            if (acc > 0.0)
                res = log10(acc) - (double)eacc * 0.30102999566398119521 - log10((double)kScale) - log10(beta);
            if (GCP && !(beta > 0.0)) res = NAN;
            v.scores[task.out] = (float)res;
            if (to_ext && !fuse) {
                const int cls = fp64_class(L);
                const unsigned long long slot = atomicAdd(ext.count + cls, 1ull);
                ext.base[ext.off[cls] + (long long)slot] = task;
            }
        }
        if (MT && !EXT && fuse) return __any_sync(kFullMask, to_ext);
        return false;
    }
};

}  // namespace phmm
