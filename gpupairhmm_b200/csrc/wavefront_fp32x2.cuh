// Packed FP32 wavefront: one group of G lanes computes two pairs that share a
// haplotype -- (read A, hap) and (read B, hap) -- with sm_100 packed FP32
// instructions (FFMA2 / FADD2 / FMUL2 on float2 register pairs).
//
// The recurrence, scaling and result carry are those of wavefront_fp32.cuh
// (I, D and the diagonal sum kept divided by their input weights: four FFMA
// and one FMUL per cell); every value is a float2 (x = read A, y = read B).
// Because both pairs see the same haplotype letter at every step, their
// lambda' values can be interleaved when the table is built: a 16-byte shared
// load returns (lam'_A(c), lam'_B(c), lam'_A(c+1), lam'_B(c+1)), i.e. the
// operands of two packed cells with no register moves.  Per cell that is 2.5
// packed FP32 instructions (the FMA-pipe cycles of 5 scalar ones, half the
// issue slots), 1/4 shared load, and 7 shuffles per step for two pairs.
// Single tile only (read length <= G*R); longer reads use the scalar kernel.
#pragma once

#include "device_common.cuh"

namespace phmm {

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

template <int G, int R>
struct Fp32x2Wavefront {
    static_assert(R % 2 == 0 && R >= 4, "R must be even");
    static_assert(G == 4 || G == 8 || G == 16 || G == 32, "G must divide the warp");
    static constexpr int NG = 32 / G;   // items (pairs of pairs) per warp
    static constexpr int T = G * R;
    static constexpr int Q = R / 2;     // float4 (2 positions x 2 reads) per thread per table row
    static constexpr int kTableFloat4 = 5 * Q * 32;  // per warp
    // read positions in groups of 4, the last group 2 when R % 4 == 2 (a lane then
    // starts 8-byte aligned and loads its packed words as uint2 pairs)
    static constexpr int NGRP = R / 4 + (R % 4 ? 1 : 0);
    __host__ __device__ static constexpr int group_size(int g) { return g < R / 4 ? 4 : 2; }

    __device__ __forceinline__ static void load_group(const uint32_t* rpack, int p0, int g, int L, uint32_t (&ws)[4]) {
        ws[0] = ws[1] = ws[2] = ws[3] = 0u;
        const int p = p0 + 4 * g;
        if (p >= L) return;
        if (g < R / 4) {
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

    __device__ __forceinline__ static void params(const DevView& v, const uint32_t* rpack, int L, int p0, const float* ph,
                                  float (&a_cur)[R], float& a_next) {
#pragma unroll
        for (int g = 0; g < NGRP; ++g) {
            uint32_t ws[4];
            load_group(rpack, p0, g, L, ws);
#pragma unroll
            for (int s = 0; s < group_size(g); ++s) {
                const int r = 4 * g + s;
                a_cur[r] = (p0 + r < L) ? 1.0f - (ph[(ws[s] >> 16) & 0x7fu] + ph[(ws[s] >> 24) & 0x7fu]) : 1.0f;
            }
        }
        a_next = 1.0f;
        if (p0 + R < L) {
            const uint32_t wn = __ldg(rpack + p0 + R);
            a_next = 1.0f - (ph[(wn >> 16) & 0x7fu] + ph[(wn >> 24) & 0x7fu]);
        }
    }

    // I scale of the position before the lane's first (1 at the read's column -1)
    __device__ __forceinline__ static float scale_before(const uint32_t* rpack, int L, int p0, const float* ph) {
        if (p0 == 0) return 1.0f;
        if (p0 - 1 >= L) return kBeta;
        const uint32_t wp = __ldg(rpack + p0 - 1);
        const float dp = ph[(wp >> 16) & 0x7fu];
        return (kBeta * dp) / (1.0f - (dp + ph[(wp >> 24) & 0x7fu]));
    }

    // one read position of one side: lambda' for the 5 haplotype codes and the
    // (q_{c-1}, e, r) coefficients (see wavefront_fp32.cuh); qp carries the I
    // scale from one position to the next
    __device__ __forceinline__ static void position(uint32_t w, int L, int c, float ac, float an, const float* ph,
                                                    float (&lam)[5], float& dv, float& ev, float& rv, float& qp,
                                                    bool& deg) {
        const uint32_t x = w & 0xffu;
        const float p = ph[(w >> 8) & 0x7fu];
        const float d = ph[(w >> 16) & 0x7fu];
        const float sgm = ph[(w >> 24) & 0x7fu];
        const bool in = c < L;
        const float lm = 1.0f - p;   // pairhmm_kernels.cuh:1244
        const float lx = p / 3.0f;   // pairhmm_kernels.cuh:1250
#pragma unroll
        for (int h = 0; h < 5; ++h) lam[h] = in ? an * ((x == 4u || h == 4 || x == (uint32_t)h) ? lm : lx) : 0.0f;
        if (in && !(fabsf(ac) >= kMinAlpha)) deg = true;
        const float qc = in ? (kBeta * d) / ac : kBeta;
        dv = qp;
        ev = ((in ? kEps : 1.0f) * qp) / qc;
        rv = in ? ((kBeta * sgm) / an) / qc : 0.0f;
        qp = qc;
    }

    __device__ static void run(const DevView& v, const Item* items, int nitem, float4* wtab, const float* ph) {
        const int lane = threadIdx.x & 31;
        const int grp = lane / G;
        const int t = lane - grp * G;
        const bool active = grp < nitem;
        const Item it = items[active ? grp : 0];
        const bool hasB = it.read1 >= 0;
        const int ra = it.read0, rb = hasB ? it.read1 : it.read0;
        const int LA = v.read_len[ra], LB = v.read_len[rb];
        const int H = v.hap_len[it.hap];
        const bool validA = active && LA >= 1 && H >= 1;
        const bool validB = validA && hasB && LB >= 1;
        const int LAc = LA >= 1 ? LA : 1, LBc = LB >= 1 ? LB : 1;
        const int Hc = H >= 1 ? H : 1;
        const uint32_t* rpA = v.read_pack + v.read_start[ra];
        const uint32_t* rpB = v.read_pack + v.read_start[rb];
        const uint32_t* hw = reinterpret_cast<const uint32_t*>(v.hap_code + v.hap_start[it.hap]);
        const float Dbound = kBeta * (kScale / (float)Hc);
        const int p0 = t * R;

        // ---------------- parameters (O(R) per lane) ----------------
        float aA[R], aB[R], anA, anB;
        params(v, rpA, LAc, p0, ph, aA, anA);
        params(v, rpB, LBc, p0, ph, aB, anB);
        bool degA = false, degB = false;
        float2 dpv[R], ee[R], rr[R], N[R], D[R];
        float qpA = scale_before(rpA, LAc, p0, ph), qpB = scale_before(rpB, LBc, p0, ph);
#pragma unroll
        for (int q = 0; q < NGRP; ++q) {
            uint32_t was[4], wbs[4];
            load_group(rpA, p0, q, LAc, was);
            load_group(rpB, p0, q, LBc, wbs);
            float lamA[5][4], lamB[5][4];
#pragma unroll
            for (int s = 0; s < group_size(q); ++s) {
                const int r = 4 * q + s;
                const int c = p0 + r;
                const float anA_r = (r + 1 < R) ? aA[r + 1 < R ? r + 1 : r] : anA;
                const float anB_r = (r + 1 < R) ? aB[r + 1 < R ? r + 1 : r] : anB;
                float la[5], lb[5];
                position(was[s], LA, c, aA[r], anA_r, ph, la, dpv[r].x, ee[r].x, rr[r].x, qpA, degA);
                position(wbs[s], LB, c, aB[r], anB_r, ph, lb, dpv[r].y, ee[r].y, rr[r].y, qpB, degB);
#pragma unroll
                for (int hh = 0; hh < 5; ++hh) {
                    lamA[hh][s] = la[hh];
                    lamB[hh][s] = lb[hh];
                }
                N[r] = f2(0.f, 0.f);
                D[r] = f2(0.f, 0.f);
            }
#pragma unroll
            for (int hh = 0; hh < 5; ++hh) {
                wtab[(hh * Q + 2 * q) * 32 + lane] = make_float4(lamA[hh][0], lamB[hh][0], lamA[hh][1], lamB[hh][1]);
                if (group_size(q) == 4)
                    wtab[(hh * Q + 2 * q + 1) * 32 + lane] =
                        make_float4(lamA[hh][2], lamB[hh][2], lamA[hh][3], lamB[hh][3]);
            }
        }

        // ---------------- steps ----------------
        const int relA = LAc - 1, relB = LBc - 1;
        const int trA = relA / R, rrA = relA - trA * R;
        const int trB = relB / R, rrB = relB - trB * R;
        const int kgA = Hc + trA, kgB = Hc + trB;
        const bool resA = validA && t == trA, resB = validB && t == trB;
        const bool addMA = rrA == R - 1, addMB = rrB == R - 1;
        // weight of the lane's last I^ in the result: beta in the carry, q when the
        // read ends on the lane's last position
        const float qresA = addMA ? qpA : kBeta, qresB = addMB ? qpB : kBeta;
        const int kmax = (int)__reduce_max_sync(kFullMask, (unsigned)(validA ? (kgA > kgB ? kgA : kgB) : 0));
        const int K = (kmax + 1 + 3) & ~3;

        const float2 k01 = f2(kEps, kEps);
        float2 Ml = f2(0.f, 0.f), Mul = Ml, Iul = Ml, Xul = Ml;
        if (t == 0) Xul = f2(Dbound, Dbound);
        double accdA = 0.0, accdB = 0.0;  // result sums: 4-step FP32 blocks added in double
        int h = 4;

        const int wlast = ((Hc + 15) & ~15) / 4 - 1;
        uint32_t wcur = __ldg(hw);
        uint32_t wnext = __ldg(hw + 1);
        for (int k0 = 0; k0 < K; k0 += 4) {
            const uint32_t wpref = __ldg(hw + min_i((k0 >> 2) + 2, wlast));
            float accA = 0.f, accB = 0.f;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int k = k0 + s;
                int hn = __shfl_up_sync(kFullMask, h, 1, G);
                if (t == 0) hn = (int)((wcur >> (8 * s)) & 0xffu);
                h = hn;
                const float4* trow = wtab + h * (Q * 32) + lane;
                float2 Nd = Mul, Id = Iul, Xd = Xul;
#pragma unroll
                for (int qq = 0; qq < Q; ++qq) {
                    const float4 lam = trow[qq * 32];
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const int r = 2 * qq + u;
                        const float2 l2 = u ? f2(lam.z, lam.w) : f2(lam.x, lam.y);
                        const float2 No = N[r];
                        const float2 Do = D[r];
                        N[r] = __fmul2_rn(l2, __ffma2_rn(dpv[r], Xd, Nd));
                        D[r] = __ffma2_rn(k01, Do, No);
                        const float2 In = __ffma2_rn(ee[r], Id, Nd);
                        Xd = __ffma2_rn(rr[r], Do, In);
                        Nd = No;
                        Id = In;
                    }
                }
                if (resA && k <= kgA) {
                    accA = fmaf(qresA, Id.x, accA);
                    if (addMA && k < kgA) accA = fmaf(kBeta, N[R - 1].x, accA);
                }
                if (resB && k <= kgB) {
                    accB = fmaf(qresB, Id.y, accB);
                    if (addMB && k < kgB) accB = fmaf(kBeta, N[R - 1].y, accB);
                }
                Mul = Ml;
                Ml = f2(__shfl_up_sync(kFullMask, N[R - 1].x, 1, G), __shfl_up_sync(kFullMask, N[R - 1].y, 1, G));
                Iul = f2(__shfl_up_sync(kFullMask, Id.x, 1, G), __shfl_up_sync(kFullMask, Id.y, 1, G));
                Xul = f2(__shfl_up_sync(kFullMask, Xd.x, 1, G), __shfl_up_sync(kFullMask, Xd.y, 1, G));
                if (t == 0) {
                    Ml = f2(0.f, 0.f);
                    Iul = f2(0.f, 0.f);
                    Xul = f2(Dbound, Dbound);
                }
            }
            if (resA) accdA += (double)accA;
            if (resB) accdB += (double)accB;
            wcur = wnext;
            wnext = wpref;
        }

        // degenerate alpha anywhere in a read's group sends that pair to FP64
        const unsigned gmask = (G == 32 ? kFullMask : ((1u << G) - 1u)) << (grp * G);
        degA = (__ballot_sync(kFullMask, degA) & gmask) != 0u;
        degB = (__ballot_sync(kFullMask, degB) & gmask) != 0u;
        const double off = log10((double)kScale) + log10((double)kBeta);
        if (resA) {
            v.scores[it.out0] = (float)(log10(accdA) - off);
            if (degA || (v.rescue_enabled && !(accdA >= (double)rescue_threshold(LA, H) && accdA <= (double)FLT_MAX))) {
                append_rescue(v, fp64_class(LA), Task{ra, it.hap, it.out0});
            }
        }
        if (resB) {
            v.scores[it.out1] = (float)(log10(accdB) - off);
            if (degB || (v.rescue_enabled && !(accdB >= (double)rescue_threshold(LB, H) && accdB <= (double)FLT_MAX))) {
                append_rescue(v, fp64_class(LB), Task{rb, it.hap, it.out1});
            }
        }
    }
};

}  // namespace phmm
