/*
 * PairHMM forward oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the CPU restatement of the reference's forward algorithm that the
 * test-suite, the smoke check and the CPU-baseline leg of bench.py compare the
 * CUDA path against.  Nothing in the product library links, loads or calls it.
 *
 * What it restates (reference = asbschmidt/gpuPairHMM):
 *   - probability table p(q) = float(10^(-q/10))            gpuworker.cuh:473-486
 *   - base encoding A,C,G,T -> 0..3, anything else -> 4      utility_kernels.cuh:6-23
 *   - emission lambda: read==hap or either is N -> 1-p(bq),
 *     otherwise p(bq)/3 (float arithmetic)                   pairhmm_kernels.cuh:1209-1262
 *   - delta=p(iq), sigma=p(dq), alpha=1-(delta+sigma),
 *     eps=0.1f, beta=0.9f (gcp is not used on the GPU path) pairhmm_kernels.cuh:1195-1196,1305-1355
 *     gcp mode (the product's option): eps=p(gcp), beta=float(1.0-eps) with
 *     gcp the read's first gcp quality, as the reference's CPU path forms
 *     them                                                   gpuworker.cuh:1009,1048-1049
 *   - D boundary = (FLT_MAX/16)/hapLength, M=I=0           pairhmm_kernels.cuh:1201,1673-1674
 *                                                           gpuworker.cuh:1034-1046
 *   - recurrence (row = read position, column = hap position)
 *       M[r][c] = lambda*(alpha*M[r-1][c-1] + beta*(I[r-1][c-1] + D[r-1][c-1]))
 *       I[r][c] = delta*M[r-1][c] + eps*I[r-1][c]
 *       D[r][c] = sigma*M[r][c-1] + eps*D[r][c-1]           gpuworker.cuh:1048-1075
 *   - result = log10(sum_c M[L][c]+I[L][c]) - log10(FLT_MAX/16)
 *                                                           gpuworker.cuh:1093-1095,
 *                                                           pairhmm_kernels.cuh:1760-1764
 *   - output slot of pair (record, read r, hap h) =
 *       sum_{previous records} R*H + r*H + h                gpuworker.cuh:1002-1021
 *
 * Arithmetic: the per-position parameters are formed exactly as the reference
 * kernel forms them (float), the recurrence runs in double.  Each block of 16
 * columns of a read row carries its own power-of-two exponent: a block is
 * computed at the largest exponent among its inputs (the others are scaled
 * down to it exactly) and renormalised when its maximum leaves [2^-100,
 * 2^100].  Pairs far below the double range, and rows whose values span more
 * than it (long haplotypes with costly gaps), still get a finite, accurate
 * log10.  Scaling is exact because the recurrence is linear.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static float g_ph2pr[128];
static int g_ph2pr_ready = 0;

static void ph2pr_init(void) {
    if (g_ph2pr_ready) return;
    for (int i = 0; i < 128; ++i) g_ph2pr[i] = (float)pow(10.0, (-i) / 10.0);
    g_ph2pr_ready = 1;
}

/* Column block width of the scaled rows and the exponent of an all-zero block.
 * Each block of a row carries its own power-of-two exponent, so values far
 * apart along a row (a deletion chain decays by eps per column: 10^-12,000
 * over 3,000 columns at eps = 1e-4) keep their range; inside a block the
 * values span at most eps^(BW-1) times the block's renormalisation band. */
#define BW 16
static const int kZeroExp = -(1 << 28);

/* 2^x for x <= 0 as an exact double (0 below the normal range: such a term is
 * below the rounding of the values it is added to) */
static inline double pow2i(int x) {
    if (x < -1022) return 0.0;
    const uint64_t bits = (uint64_t)(x + 1023) << 52;
    double d;
    memcpy(&d, &bits, sizeof d);
    return d;
}

/* quality bytes index a 128-entry table; larger values are clamped to 127 */
static inline float ph2pr(uint8_t q) { return g_ph2pr[q > 127 ? 127 : q]; }

/* utility_kernels.cuh:6-23 */
int oracle_encode_base(uint8_t c) {
    switch (c) {
        case 'A': return 0;
        case 'C': return 1;
        case 'G': return 2;
        case 'T': return 3;
        default: return 4;
    }
}

float oracle_ph2pr(int q) {
    ph2pr_init();
    return ph2pr((uint8_t)(q < 0 ? 0 : (q > 255 ? 255 : q)));
}

/*
 * One pair.  Returns log10 likelihood (double).  read/hap are ASCII bases,
 * quals are Phred values (ASCII already minus 33).  L >= 1 and H >= 1.
 * gcp < 0: eps = 0.1f, beta = 0.9f (the reference's GPU path); gcp >= 0:
 * eps = p(gcp), beta = float(1 - eps) (its CPU path, gpuworker.cuh:1048-1049).
 * Work buffer: 3*(H+1) doubles x 2 rows, allocated here.
 */
double oracle_pair_log10_gcp(const uint8_t* read, const uint8_t* bq, const uint8_t* iq,
                             const uint8_t* dq, int L, const uint8_t* hap, int H, int gcp) {
    ph2pr_init();
    if (L <= 0 || H <= 0) return NAN;
    const float constant_f = FLT_MAX / 16.0f;
    const float initD_f = constant_f / (float)H;
    const float eps_f = gcp < 0 ? 0.1f : ph2pr((uint8_t)(gcp > 255 ? 255 : gcp));
    const float beta_f = gcp < 0 ? 0.9f : (float)(1.0 - (double)eps_f);
    const double beta = (double)beta_f;
    const double eps = (double)eps_f;
    const int nb = (H + BW - 1) / BW; /* column blocks over columns 1..H */

    double* buf = (double*)malloc(sizeof(double) * 6 * (size_t)(H + 1));
    double *Mp = buf, *Ip = buf + (H + 1), *Dp = buf + 2 * (H + 1);
    double *Mc = buf + 3 * (H + 1), *Ic = buf + 4 * (H + 1), *Dc = buf + 5 * (H + 1);
    int* Ep = (int*)malloc(sizeof(int) * 2 * (size_t)nb);
    int* Ec = Ep + nb;
    int* hcode = (int*)malloc(sizeof(int) * (size_t)H);
    for (int c = 0; c < H; ++c) hcode[c] = oracle_encode_base(hap[c]);

    /* row "-1": M = I = 0, D = initD for every column (gpuworker.cuh:1041-1044) */
    for (int c = 0; c <= H; ++c) { Mp[c] = 0.0; Ip[c] = 0.0; Dp[c] = (double)initD_f; }
    for (int k = 0; k < nb; ++k) Ep[k] = 0;
    int ecol0 = 0; /* exponent of column 0 of the previous row (nonzero only in row -1) */

    for (int r = 0; r < L; ++r) {
        const float p = ph2pr(bq[r]);
        const float lam_match = 1.0f - p;
        const float lam_mis = p / 3.0f;
        const float delta_f = ph2pr(iq[r]);
        const float sigma_f = ph2pr(dq[r]);
        const float alpha_f = 1.0f - (delta_f + sigma_f);
        const double delta = delta_f, sigma = sigma_f, alpha = alpha_f;
        const int x = oracle_encode_base(read[r]);
        /* emission by haplotype code for this read position */
        double lamtab[5];
        for (int hh = 0; hh < 5; ++hh)
            lamtab[hh] = (x == 4 || hh == 4 || x == hh) ? (double)lam_match : (double)lam_mis;

        Mc[0] = 0.0; Ic[0] = 0.0; Dc[0] = 0.0;
        for (int k = 0; k < nb; ++k) {
            const int c0 = 1 + k * BW, c1 = c0 + BW - 1 < H ? c0 + BW - 1 : H;
            /* the block takes the largest exponent among its inputs; the others
               are scaled down to it by exact powers of two */
            const int epl = k ? Ep[k - 1] : ecol0; /* previous row, column c0-1 */
            const int ecl = k ? Ec[k - 1] : kZeroExp; /* this row, column c0-1 */
            int e = Ep[k];
            if (epl > e) e = epl;
            if (ecl > e) e = ecl;
            const double fp = pow2i(Ep[k] - e), fpl = pow2i(epl - e), fcl = pow2i(ecl - e);
            double mdiag = Mp[c0 - 1] * fpl, idiag = Ip[c0 - 1] * fpl, ddiag = Dp[c0 - 1] * fpl;
            double mleft = Mc[c0 - 1] * fcl, dleft = Dc[c0 - 1] * fcl;
            double bmax = 0.0;
            if (fp == 1.0) { /* the block keeps its exponent: no scaling inside */
                for (int c = c0; c <= c1; ++c) {
                    const double lam = lamtab[hcode[c - 1]];
                    const double m = lam * (alpha * mdiag + beta * (idiag + ddiag));
                    const double i = delta * Mp[c] + eps * Ip[c];
                    const double d = sigma * mleft + eps * dleft;
                    mdiag = Mp[c]; idiag = Ip[c]; ddiag = Dp[c];
                    Mc[c] = m; Ic[c] = i; Dc[c] = d;
                    mleft = m; dleft = d;
                    double v = m > i ? m : i;
                    v = v > d ? v : d;
                    if (v > bmax) bmax = v;
                }
            } else {
                for (int c = c0; c <= c1; ++c) {
                    const double lam = lamtab[hcode[c - 1]];
                    const double mup = Mp[c] * fp, iup = Ip[c] * fp;
                    const double m = lam * (alpha * mdiag + beta * (idiag + ddiag));
                    const double i = delta * mup + eps * iup;
                    const double d = sigma * mleft + eps * dleft;
                    mdiag = mup; idiag = iup; ddiag = Dp[c] * fp;
                    Mc[c] = m; Ic[c] = i; Dc[c] = d;
                    mleft = m; dleft = d;
                    double v = m > i ? m : i;
                    v = v > d ? v : d;
                    if (v > bmax) bmax = v;
                }
            }
            Ec[k] = e;
            if (bmax == 0.0) {
                Ec[k] = kZeroExp;
            } else if (bmax < 0x1p-100 || bmax > 0x1p+100) {
                /* exact power-of-two renormalisation of the block */
                int be;
                frexp(bmax, &be);
                for (int c = c0; c <= c1; ++c) {
                    Mc[c] = ldexp(Mc[c], -be); Ic[c] = ldexp(Ic[c], -be); Dc[c] = ldexp(Dc[c], -be);
                }
                Ec[k] = e + be;
            }
        }
        ecol0 = kZeroExp;
        double* t;
        t = Mp; Mp = Mc; Mc = t;
        t = Ip; Ip = Ic; Ic = t;
        t = Dp; Dp = Dc; Dc = t;
        int* te = Ep; Ep = Ec; Ec = te;
    }
    /* sum_c (M+I) of the last row, block sums brought to the largest exponent */
    int emax = kZeroExp;
    for (int k = 0; k < nb; ++k)
        if (Ep[k] > emax) emax = Ep[k];
    double sum = 0.0;
    if (emax > kZeroExp) {
        for (int k = 0; k < nb; ++k) {
            const int c0 = 1 + k * BW, c1 = c0 + BW - 1 < H ? c0 + BW - 1 : H;
            double s = 0.0;
            for (int c = c0; c <= c1; ++c) s += Mp[c] + Ip[c];
            sum += s * pow2i(Ep[k] - emax);
        }
    }
    free(buf);
    free(hcode);
    free(Ep < Ec ? Ep : Ec);
    if (!(sum > 0.0)) return -INFINITY;
    return log10(sum) + (double)emax * log10(2.0) - log10((double)constant_f);
}

double oracle_pair_log10(const uint8_t* read, const uint8_t* bq, const uint8_t* iq,
                         const uint8_t* dq, int L, const uint8_t* hap, int H) {
    return oracle_pair_log10_gcp(read, bq, iq, dq, L, hap, H, -1);
}

/*
 * Whole batch in the reference's record layout.  Output slot order follows
 * gpuworker.cuh:1002-1021 (record-major, then read, then haplotype).
 * Offsets are per read / per haplotype start indices into the byte arrays.
 * nthreads <= 0 uses the OpenMP default.  Returns the number of pairs.
 */
/* gcp_quals == NULL: the GPU path's eps and beta; else each read takes its
 * first position's gcp quality (gpuworker.cuh:1009). */
int64_t oracle_batch_log10_gcp(int64_t num_records, const int32_t* reads_per_record,
                               const int32_t* haps_per_record, const uint8_t* read_bases,
                               const uint8_t* base_quals, const uint8_t* ins_quals,
                               const uint8_t* del_quals, const uint8_t* gcp_quals,
                               const int64_t* read_offsets, const int32_t* read_lengths,
                               const uint8_t* hap_bases, const int64_t* hap_offsets,
                               const int32_t* hap_lengths, double* out, int nthreads) {
    ph2pr_init();
    /* per-record prefix sums of reads, haps and pairs */
    int64_t* rp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(num_records + 1) * 3);
    int64_t *hp = rp + (num_records + 1), *pp = rp + 2 * (num_records + 1);
    rp[0] = hp[0] = pp[0] = 0;
    for (int64_t g = 0; g < num_records; ++g) {
        rp[g + 1] = rp[g] + reads_per_record[g];
        hp[g + 1] = hp[g] + haps_per_record[g];
        pp[g + 1] = pp[g] + (int64_t)reads_per_record[g] * haps_per_record[g];
    }
    const int64_t npairs = pp[num_records];
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t pidx = 0; pidx < npairs; ++pidx) {
        /* record by binary search over pair prefix sums */
        int64_t lo = 0, hi = num_records;
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) / 2;
            if (pp[mid] <= pidx) lo = mid; else hi = mid;
        }
        while (lo < num_records && pp[lo + 1] <= pidx) ++lo;
        const int64_t g = lo;
        const int64_t local = pidx - pp[g];
        const int H = haps_per_record[g];
        const int64_t r = rp[g] + local / H;
        const int64_t h = hp[g] + local % H;
        const int64_t ro = read_offsets[r], ho = hap_offsets[h];
        out[pidx] = oracle_pair_log10_gcp(read_bases + ro, base_quals + ro, ins_quals + ro,
                                          del_quals + ro, read_lengths[r], hap_bases + ho,
                                          hap_lengths[h], gcp_quals ? (int)gcp_quals[ro] : -1);
    }
    free(rp);
    return npairs;
}

int64_t oracle_batch_log10(int64_t num_records, const int32_t* reads_per_record,
                           const int32_t* haps_per_record, const uint8_t* read_bases,
                           const uint8_t* base_quals, const uint8_t* ins_quals,
                           const uint8_t* del_quals, const int64_t* read_offsets,
                           const int32_t* read_lengths, const uint8_t* hap_bases,
                           const int64_t* hap_offsets, const int32_t* hap_lengths,
                           double* out, int nthreads) {
    return oracle_batch_log10_gcp(num_records, reads_per_record, haps_per_record, read_bases,
                                  base_quals, ins_quals, del_quals, NULL, read_offsets,
                                  read_lengths, hap_bases, hap_offsets, hap_lengths, out, nthreads);
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
