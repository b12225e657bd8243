// FP32 anti-diagonal wavefront for the PairHMM forward recurrence.
//
// Work split (one warp = 32/G groups, one pair per group):
//   lane t of a group owns R consecutive read positions c = tile*T + t*R + r,
//   T = G*R.  Haplotype positions stream through the group: at step k lane t
//   works on haplotype row j = k - t, so the group sweeps one anti-diagonal
//   band per step.  The last N, D and I of a lane move one lane up with
//   __shfl_up_sync each step (the boundary column hand-off).
//
// Recurrence (the algebra of pairhmm_kernels.cuh:1417-1651 and
// gpuworker.cuh:1048-1075):
//     M(j,c) = lambda(h_j,c) * (alpha_c*M(j-1,c-1) + beta*(I(j-1,c-1) + D(j-1,c-1)))
//     I(j,c) = delta_c*M(j,c-1) + eps*I(j,c-1)
//     D(j,c) = sigma_c*M(j-1,c) + eps*D(j-1,c)
// stored in rescaled variables that fold every constant factor into tables:
//     N = alpha_{c+1}*M,  It = beta*I,  Dt = beta*D
//     N(j,c)  = lam'(h_j,c) * (N(j-1,c-1) + It(j-1,c-1) + Dt(j-1,c-1)),  lam' = alpha_{c+1}*lambda
//     It(j,c) = d'_c*N(j,c-1) + eps_c*It(j,c-1),                        d'   = beta*delta_c/alpha_c
//     Dt(j,c) = s'_c*N(j-1,c) + eps*Dt(j-1,c),                          s'   = beta*sigma_c/alpha_{c+1}
// and each of It and Dt divided by its own per-position input weight, so that
// the term that feeds it has weight 1 and folds into an FFMA:
//     I^ = It/q_c  (q_c = d'_c inside the read, beta from the read end on),
//     D^ = Dt/s'_c,  X^ = (It + Dt(j-1))/q_c  (the diagonal sum N needs):
//     D^(j,c) = eps*D^(j-1,c) + N(j-1,c)                        FFMA
//     I^(j,c) = e_c*I^(j,c-1) + N(j-1,c-1)                      FFMA  e_c = eps_c*q_{c-1}/q_c
//     X^(j,c) = r_c*D^(j-1,c) + I^(j,c)                         FFMA  r_c = s'_c/q_c
//     N(j,c)  = lam'(h_j,c) * (q_{c-1}*X^(j,c-1) + N(j-1,c-1))   FFMA + FMUL
// Five FP32 instructions per cell (four FFMA, one FMUL), only lam' (4 bytes
// per cell) from shared memory, and per-position registers N, D^, q_{c-1},
// e, r (5R).  The rescaled values stay on the scale of N (q and s' are the
// weights of what feeds them), so the FP32 range is that of the unscaled
// form.  Pairs with |alpha| < 2^-8 somewhere (ins+del quality around 3 or
// below) cannot use the division; they are flagged for the FP64 pass, which
// runs the untransformed recurrence.  I is computed one anti-diagonal behind
// M, as in the reference (pairhmm_kernels.cuh:1423-1426).
//
// Result: positions from the read end on take eps = 1 and the scale q = beta
// (so N(j-1, L-1) enters I at L with weight beta and later positions only
// carry); beta times the lane's last I^ is then beta*(M+I)(j, L-1) (the
// reference's trick, pairhmm_kernels.cuh:1307-1331, with beta folded in).
// When the read ends on a lane's last position the lane adds q*I^ + beta*N.
// Summing over j gives beta * sum_j (M+I)(L-1,j).  The sum runs over up to
// H rows of similar size, which in FP32 alone drifts by up to ~H*2^-25
// relative (1e-4 at H = 16384); each block of 4 steps is summed in FP32 and
// the blocks in double, so it is exact to well below the output's precision.
//
// lam' table: each thread owns 5 x R floats in shared memory, laid out as
// [hap code][R/4][32 lanes] float4, so a warp-wide 16-byte load touches 32
// consecutive float4s whatever codes the lanes hold (no bank conflicts) and a
// thread only reads what it wrote (no synchronisation).  With R % 4 == 2 the
// last two positions of each code follow as a [hap code][32 lanes] float2
// table (a 150-position read fits 8 x 18 = 144 + one more tile row instead of
// 8 x 20 = 160: fewer padded cells for the common 129-144 lengths).
//
// GCP = true (gcp mode): eps and beta are the read's own instead of the
// constants; everything else is the same.
//
// Reads longer than T (MT = true) run as several tiles; the last lane of tile
// i writes (X^, I^, N) of its last position for every haplotype row into a
// per-group scratch border, which lane 0 of tile i+1 reads as its left
// boundary (pairhmm_kernels.cuh:2167-3272 does the same with 512-row tiles).
// The group's lanes fetch those rows G at a time from L2 one block ahead and
// put them in a per-warp shared ring, from which each step takes its row with
// one broadcast load (three shuffles per step before).
//
// Early hand-off of long pairs that will underflow: every path to the result
// crosses the border column once, and transitions and emissions never exceed
// 1, so the final sum is at most the mass on the border, sum_j (M+I+D)(j).
// After each tile but the last the group adds up its border rows (in L2, a
// few loads per lane); when that mass is below half the FP64 threshold the
// final sum would be below the threshold too, so the pair is flagged for the
// FP64 pass at once and its remaining tiles are skipped.  Which pairs the
// FP64 pass recomputes, and so every result, is unchanged; long unrelated
// reads no longer run their later FP32 tiles for nothing.
#pragma once

#include "device_common.cuh"

namespace phmm {

template <int G, int R, bool MT, bool GCP = false>
struct Fp32Wavefront {
    static_assert(R % 2 == 0 && R >= 4, "R must be even");
    static_assert(G == 4 || G == 8 || G == 16 || G == 32, "G must divide the warp");
    static constexpr int NG = 32 / G;   // pairs per warp
    static constexpr int T = G * R;     // read positions per tile
    static constexpr int Q = R / 4;     // float4 per thread per table row
    static constexpr bool kTail = R % 4 == 2;       // then one float2 group after them
    static constexpr int NGRP = Q + (kTail ? 1 : 0);  // position groups: 4 each, the tail 2
    static constexpr int kTail2 = 5 * Q * 32;       // float4 index where the float2 tail table starts
    static constexpr int kLamFloat4 = 5 * Q * 32 + (kTail ? 5 * 32 / 2 : 0);
    // per warp: the lam' table, then (MT) a 32-entry ring of border rows
    static constexpr int kTableFloat4 = kLamFloat4 + (MT ? 32 : 0);

    __host__ __device__ static constexpr int group_size(int g) { return g < Q ? 4 : 2; }

    // Packed words of position group g of the lane starting at p0 (zero past the
    // read's padded end).  A lane starts at a multiple of R positions, so with
    // R % 4 == 2 its groups are only 8-byte aligned and load as uint2 pairs.
    __device__ __forceinline__ static void load_group(const uint32_t* rpack, int p0, int g, int Lc,
                                                      uint32_t (&ws)[4]) {
        ws[0] = ws[1] = ws[2] = ws[3] = 0u;
        const int p = p0 + 4 * g;
        if (p >= Lc) return;
        if (g < Q) {
            if constexpr (R % 4 == 0) {
                const uint4 w = __ldg(reinterpret_cast<const uint4*>(rpack + p));
                ws[0] = w.x; ws[1] = w.y; ws[2] = w.z; ws[3] = w.w;
            } else {
                const uint2 a = __ldg(reinterpret_cast<const uint2*>(rpack + p));
                const uint2 b = __ldg(reinterpret_cast<const uint2*>(rpack + p + 2));
                ws[0] = a.x; ws[1] = a.y; ws[2] = b.x; ws[3] = b.y;
            }
        } else {
            const uint2 a = __ldg(reinterpret_cast<const uint2*>(rpack + p));
            ws[0] = a.x; ws[1] = a.y;
        }
    }

    // items: the warp's ntask (<= NG) work items (read1 unused).  wtab: this warp's table
    // (kTableFloat4 float4).  ph: 128-entry probability table (shared).
    // scratch: this warp's border storage, NG groups x 2 buffers x rows float4.
    __device__ static void run(const DevView& v, const Item* items, int ntask, float4* wtab,
                               const float* ph, float4* scratch, int64_t rows) {
        const int lane = threadIdx.x & 31;
        const int grp = lane / G;
        const int t = lane - grp * G;
        const bool active = grp < ntask;
        const Item it = items[active ? grp : 0];
        const Task task{it.read0, it.hap, it.out0};  // units of this kernel hold one read
        const int L = v.read_len[task.read];
        const int H = v.hap_len[task.hap];
        const bool valid = active && L >= 1 && H >= 1;
        const int Lc = L >= 1 ? L : 1;
        const int Hc = H >= 1 ? H : 1;
        const int ntiles = MT ? (Lc + T - 1) / T : 1;
        const int nt_warp = MT ? (int)__reduce_max_sync(kFullMask, (unsigned)ntiles) : 1;

        const uint32_t* rpack = v.read_pack + v.read_start[task.read];
        const uint32_t* hw = reinterpret_cast<const uint32_t*>(v.hap_code + v.hap_start[task.hap]);
        // eps and beta: the reference GPU path's constants, or in gcp mode the
        // read's own from its first gcp quality, formed as the reference's CPU
        // recurrence forms them (gpuworker.cuh:1048-1049)
        const float eps = GCP ? ph[v.read_gcp[task.read]] : kEps;
        const float beta = GCP ? (float)(1.0 - (double)eps) : kBeta;
        const float Dbound = beta * (kScale / (float)Hc);

        double accd = 0.0;       // result sum: 4-step FP32 blocks added in double
        int rlane = -1;          // lane (in group) that holds the result
        bool degenerate = false; // some |alpha| < kMinAlpha: FP64 pass recomputes the pair
        if (GCP && !(beta >= kMinAlpha)) degenerate = true;  // gcp quality 0: nothing to rescale by

        bool handed_off = false;  // MT: flagged for the FP64 pass at a tile border
        for (int tile = 0; tile < nt_warp; ++tile) {
            const bool tile_live = valid && !handed_off && tile < ntiles;
            const bool last = tile == ntiles - 1;
            const int p0 = tile * T + t * R;

            // ---------------- per-tile parameters (O(R) per lane) ----------------
            // alpha of the position after this lane's last one (next lane / tile)
            float alpha_next;
            {
                const int cn = p0 + R;
                alpha_next = 1.0f;
                if (cn < Lc) {
                    const uint32_t wn = __ldg(rpack + cn);
                    alpha_next = 1.0f - (ph[(wn >> 16) & 0x7fu] + ph[(wn >> 24) & 0x7fu]);
                }
            }
            // I scale of the position before this lane's first: 1 at the read's
            // column -1 (boundary values enter unscaled)
            float q_prev = 1.0f;
            if (p0 > 0) {
                q_prev = beta;
                if (p0 - 1 < L) {
                    const uint32_t wp = __ldg(rpack + p0 - 1);
                    const float dp = ph[(wp >> 16) & 0x7fu];
                    q_prev = (beta * dp) / (1.0f - (dp + ph[(wp >> 24) & 0x7fu]));
                }
            }
            float dpv[R], ee[R], rr[R];
            float N[R], D[R];
            float a_cur[R];
#pragma unroll
            for (int g = 0; g < NGRP; ++g) {
                uint32_t ws[4];
                load_group(rpack, p0, g, Lc, ws);
#pragma unroll
                for (int s = 0; s < group_size(g); ++s) {
                    const int r = 4 * g + s;
                    const float d = ph[(ws[s] >> 16) & 0x7fu];
                    const float sg = ph[(ws[s] >> 24) & 0x7fu];
                    a_cur[r] = (p0 + r < L) ? 1.0f - (d + sg) : 1.0f;  // pairhmm_kernels.cuh:1336
                }
            }
            float qp = q_prev;
            // Single-tile kernels carry 1/alpha forward (two divisions per position instead of
            // four); the multi-tile kernel keeps the divisions, its 255-register budget spills
            // with the extra live value.
            float ia = MT ? 1.0f : 1.0f / a_cur[0];
#pragma unroll
            for (int g = 0; g < NGRP; ++g) {
                uint32_t ws[4];
                load_group(rpack, p0, g, Lc, ws);
                float lam[5][4];
#pragma unroll
                for (int s = 0; s < group_size(g); ++s) {
                    const int r = 4 * g + s;
                    const int c = p0 + r;
                    const uint32_t x = ws[s] & 0xffu;
                    const float p = ph[(ws[s] >> 8) & 0x7fu];
                    const float d = ph[(ws[s] >> 16) & 0x7fu];
                    const float sg = ph[(ws[s] >> 24) & 0x7fu];
                    const bool in = c < L;
                    const float an = (r + 1 < R) ? a_cur[r + 1 < R ? r + 1 : r] : alpha_next;
                    const float lm = 1.0f - p;      // pairhmm_kernels.cuh:1244
                    const float lx = p / 3.0f;      // pairhmm_kernels.cuh:1250
#pragma unroll
                    for (int h = 0; h < 5; ++h)
                        lam[h][s] = in ? an * ((x == 4u || h == 4 || x == (uint32_t)h) ? lm : lx) : 0.0f;
                    if (in && !(fabsf(a_cur[r]) >= kMinAlpha)) degenerate = true;
                    dpv[r] = qp;
                    if constexpr (MT) {
                        const float qc = in ? (beta * d) / a_cur[r] : beta;  // I scale of c
                        ee[r] = ((in ? eps : 1.0f) * qp) / qc;
                        rr[r] = in ? ((beta * sg) / an) / qc : 0.0f;
                        qp = qc;
                    } else {
                        const float ian = 1.0f / an;
                        const float qc = in ? (beta * d) * ia : beta;  // I scale of c
                        const float iqc = 1.0f / qc;
                        ee[r] = ((in ? eps : 1.0f) * qp) * iqc;
                        rr[r] = in ? ((beta * sg) * ian) * iqc : 0.0f;
                        qp = qc;
                        ia = ian;
                    }
                    N[r] = 0.0f;
                    D[r] = 0.0f;
                }
#pragma unroll
                for (int h = 0; h < 5; ++h) {
                    if (g < Q)
                        wtab[(h * Q + g) * 32 + lane] = make_float4(lam[h][0], lam[h][1], lam[h][2], lam[h][3]);
                    else
                        reinterpret_cast<float2*>(wtab + kTail2)[h * 32 + lane] = make_float2(lam[h][0], lam[h][1]);
                }
            }
            const float q_last = qp;  // I scale of this lane's last position

            // ---------------- steps of this tile ----------------
            int t_res = 0, r_res = 0;
            if (last) {
                const int rel = Lc - 1 - tile * T;
                t_res = rel / R;
                r_res = rel - t_res * R;
            }
            // last step index that matters for this group
            const int kg = last ? (Hc + t_res) : (Hc + G - 1);
            const bool res_lane = tile_live && last && t == t_res;
            const bool addM = r_res == R - 1;
            // weight of the lane's last I^ in the result: beta in the carry, q when
            // the read ends on the lane's last position
            const float qres = addM ? q_last : beta;
            if (res_lane) rlane = t;
            const int kmax = (int)__reduce_max_sync(kFullMask, (unsigned)(tile_live ? kg : 0));
            const int K = (kmax + 1 + 3) & ~3;

            // left-boundary inputs of the next step: N(j-1), I^(j), X^(j) of the
            // column before this lane (read column -1: X = Dt = Dbound)
            float Ml = 0.f, Mul = 0.f, Iul = 0.f, Xul = 0.f;
            if (t == 0 && tile == 0) Xul = Dbound;
            int h = 4;

            // border in/out (MT only).  Row j of a buffer sits at entry G + j: the last
            // lane writes rows k - G .. k - G + 1 at step k from k = 0 on without bounds
            // branches, rows before 0 and after the haplotype's last landing in the
            // padding (a buffer has at least max H + 72 entries; a tile's last write is
            // row H + 3, at entry H + G + 3)
            float4* ein = nullptr;
            float4* eout = nullptr;
            const int64_t nrow = rows - G;  // rows a buffer holds after the padding
            float4 bcur = make_float4(0.f, 0.f, 0.f, 0.f);  // lane t: row t of the next block of G
            if (MT) {
                float4* gbase = scratch + (int64_t)grp * 2 * rows;
                if (tile > 0) {
                    ein = gbase + ((tile - 1) & 1) * rows + G;
                    if (t < nrow) bcur = __ldcg(ein + t);
                }
                eout = gbase + (tile & 1) * rows + G;
            }
            const bool writer = MT && tile_live && !last && t == G - 1;
            float ib0 = 0.f;  // writer: I^ of row 0 on the border column

            // code words of this group's haplotype; a group whose haplotype is
            // shorter than the warp's step count keeps re-reading its last word
            // (any code there is harmless: those rows are past the haplotype)
            const int wlast = ((Hc + 15) & ~15) / 4 - 1;
            uint32_t wcur = __ldg(hw);
            uint32_t wnext = __ldg(hw + 1);
            float4* ring = wtab + kLamFloat4;  // MT: rows of the group's current block of G steps
            for (int k0 = 0; k0 < K; k0 += 4) {
                const uint32_t wpref = __ldg(hw + min_i((k0 >> 2) + 2, wlast));
                if (MT && tile > 0 && (k0 & (G - 1)) == 0) {
                    // lane t of the group holds row k0 + t: into the ring, then prefetch
                    __syncwarp();
                    ring[lane] = bcur;
                    __syncwarp();
                    const int64_t idx = (int64_t)k0 + G + t;
                    bcur = idx < nrow ? __ldcg(ein + idx) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
                float acc = 0.f;
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int k = k0 + s;
                    int hn = __shfl_up_sync(kFullMask, h, 1, G);
                    if (t == 0) hn = (int)((wcur >> (8 * s)) & 0xffu);
                    h = hn;
                    const float4* trow = wtab + h * (Q * 32) + lane;
                    float Ndiag = Mul, Idiag = Iul, Xdiag = Xul;
#pragma unroll
                    for (int g = 0; g < NGRP; ++g) {
                        float ls[4];
                        if (g < Q) {
                            const float4 lam = trow[g * 32];
                            ls[0] = lam.x; ls[1] = lam.y; ls[2] = lam.z; ls[3] = lam.w;
                        } else {
                            const float2 lam = reinterpret_cast<const float2*>(wtab + kTail2)[h * 32 + lane];
                            ls[0] = lam.x; ls[1] = lam.y; ls[2] = ls[3] = 0.0f;
                        }
#pragma unroll
                        for (int u = 0; u < group_size(g); ++u) {
                            const int r = 4 * g + u;
                            const float Nold = N[r];
                            const float Dold = D[r];
                            N[r] = ls[u] * fmaf(dpv[r], Xdiag, Ndiag);
                            D[r] = fmaf(eps, Dold, Nold);
                            // e*I^ carries the serial chain: one FFMA per position
                            const float In = fmaf(ee[r], Idiag, Ndiag);
                            Xdiag = fmaf(rr[r], Dold, In);
                            Ndiag = Nold;
                            Idiag = In;
                        }
                    }
                    // result (row k - t_res): I at the lane end, plus beta*M(j) when
                    // the read ends on the lane's last register
                    if (res_lane && k <= kg) {
                        acc = fmaf(qres, Idiag, acc);
                        if (addM && k < kg) acc = fmaf(beta, N[R - 1], acc);
                    }
                    if (MT && writer) {
                        // slot s holds X^(s+1), I^(s+1), N(s); I^(0) stays in a register
                        const int j = k - (G - 1);
                        if (j == 0) ib0 = Idiag;
                        reinterpret_cast<float*>(eout + j)[2] = N[R - 1];
                        *reinterpret_cast<float2*>(eout + (j - 1)) = make_float2(Xdiag, Idiag);
                    }
                    // boundary hand-off
                    Mul = Ml;
                    Ml = __shfl_up_sync(kFullMask, N[R - 1], 1, G);
                    Iul = __shfl_up_sync(kFullMask, Idiag, 1, G);
                    Xul = __shfl_up_sync(kFullMask, Xdiag, 1, G);
                    if (MT && tile > 0) {
                        // the border is indexed by row: it feeds the diagonal of the next
                        // step directly (lanes t > 0 get theirs through the Ml -> Mul rotation)
                        const float4 brow = ring[grp * G + (k & (G - 1))];  // broadcast within the group
                        if (t == 0) { Xul = brow.x; Iul = brow.y; Mul = brow.z; }
                    } else if (t == 0) {
                        Ml = 0.f;
                        Iul = 0.f;
                        Xul = Dbound;
                    }
                }
                if (res_lane) accd += (double)acc;
                wcur = wnext;
                wnext = wpref;
            }
            __syncwarp();
            const bool check = MT && v.rescue_enabled && tile_live && !last;
            if (MT && __any_sync(kFullMask, check)) {  // warp-uniform: every lane shuffles
                // mass on this tile's border column: slot s holds X^(s+1), I^(s+1), N(s);
                // M = N/alpha_next, I + D(j-1) = q*X^/beta and I(0) = q*I^(0)/beta at the
                // last position of lane G-1 (the sum also takes I of the row after the
                // haplotype's last, which only makes it larger)
                const int src = grp * G + G - 1;
                const float an = __shfl_sync(kFullMask, alpha_next, src);
                const float qb = __shfl_sync(kFullMask, q_last, src) / beta;
                const float i0 = __shfl_sync(kFullMask, ib0, src);
                float mass = 0.f;
                if (check) {
                    if (t == 0) mass = qb * i0;
                    for (int j = t; j < Hc; j += G) {
                        const float4 b = __ldcg(eout + j);
                        mass += b.z / an + qb * b.x;
                    }
                }
#pragma unroll
                for (int d = G / 2; d >= 1; d >>= 1) mass += __shfl_xor_sync(kFullMask, mass, d, G);
                if (check && mass < 0.5f * rescue_threshold(L, H)) handed_off = true;
            }
            if (MT && __all_sync(kFullMask, !valid || handed_off || tile + 1 >= ntiles)) break;
        }

        // any lane of the group saw a degenerate alpha
        const unsigned dmask = __ballot_sync(kFullMask, degenerate);
        const unsigned gmask = (G == 32 ? kFullMask : ((1u << G) - 1u)) << (grp * G);
        degenerate = (dmask & gmask) != 0u;
        if (valid && handed_off && t == 0) {
            v.scores[task.out] = -INFINITY;  // the FP64 pass writes the result
            append_rescue(v, fp64_class(L), task);
        }
        if (valid && !handed_off && t == rlane) {
            const float res = (float)(log10(accd) - (log10((double)kScale) + log10((double)beta)));
            v.scores[task.out] = res;
            if (degenerate ||
                (v.rescue_enabled && !(accd >= (double)rescue_threshold(L, H) && accd <= (double)FLT_MAX))) {
                append_rescue(v, fp64_class(L), task);
            }
        }
    }
};

}  // namespace phmm
