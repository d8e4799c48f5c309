// sw_kernel.cu -- batched Smith-Waterman (scores + end coordinates) for sm_100a.
//
// Result semantics: exactly those of TOPAZ's striped SSW calls
//   ssw_init(q, qlen, mat, 25, 2); ssw_align(prof, s, slen, go, ge, 0, 0, 0, 15)
// (src/ssw.c:799-897): the u8 pass, the i16 pass when the u8 pass saturates
// (max + bias >= 255), and the drop when the i16 pass reaches 32767.
//
// The striped u8/i16 passes split the query into 16 (u8) or 8 (i16) SSW
// "lanes" of seg = ceil(qlen/lanes) consecutive rows.  What they compute is
// the recurrence below (pinned against src/ssw.c by the oracle tests):
//   Hp(r,c) = max(0, H(r-1,c-1) + M[s_c][q_r], E(r,c), Fm(r,c))
//   H(r,c)  = max(Hp(r,c), F(r,c))
//   E(r,c+1)= max(E(r,c) - ge, Hp(r,c) - go)
//   Fm(r+1) = (r+1) % seg == 0 ? 0 : max(Fm(r) - ge, Hp(r) - go)
//   F(r+1)  = max(F(r) - ge, H(r) - go)
// With X = max(0, H(r-1,c-1) + M, E) and Xg = X - go, and gap_open >
// gap_extend, this is the same as
//   H = max(X, F);  Gp = max(Fm - go, Xg);  E' = max(E - ge, Gp)
//   F' = max(F - ge, Xg);  Fm' = max(Fm - ge, Xg)  (Fm cleared at SSW lane starts)
// in which the only serial dependences from row to row are the F and Fm
// chains, one DPX op each.  ref_end is the first column holding the maximum,
// read_end the smallest row holding it there (src/ssw.c:264-297).
//
// Kernel layout (B200): one warp per task of two pairs packed as int16x2
// (pair A in the low half, pair B in the high half).  Lane t owns query rows
// [t*R, t*R+R) of both pairs; subject columns stream through the lanes as a
// wavefront, lane t working on column k-t at step k, with H/F/Fm of a lane's
// last row and the subject letters handed to lane t+1 by __shfl_up_sync.
// Every cell update is a DPX instruction (__viaddmax_s16x2[_relu],
// __vimax_s16x2_relu, __vimax3_s16x2).  The int8 query profile of both pairs
// sits in shared memory in a lane-blocked layout with an odd word stride per
// lane, so the 32 per-lane loads of a step never share a bank; prmt with the
// sign-replicate selector widens two profile bytes into one int16x2 operand.
//
// End coordinates: each lane keeps the running maximum of its rows and the
// column/row where it last rose.  A rise is only looked at when it reaches
// the warp maximum of the last refresh (every 32 steps; a lower value cannot
// be the alignment's maximum), and then the whole warp finds the first row
// holding the new value with packed DPX ops, so the common case costs one
// vote per step.  Steps run two at a time, the profile words ping-ponging
// between two register sets.
//
// Pairs are binned on the device by R = ceil(qlen/32) and by subject length
// (counting sort), paired two per task within a bin, and drained by one
// persistent kernel per R from an atomic task counter.  Pairs whose u8-pass
// maximum saturates are appended to their bin's rerun list and re-run with
// the i16 lane length (seg = ceil(qlen/8)) by a second kernel of the bin on
// the same stream.  With qlen <= 1024 and |M| <= 127 no score can reach
// 32767, so 16-bit arithmetic is exact.
//
// Every lane computes every step, also before its first column and past
// the subject's end (pad letters there), so the step body has no per-lane
// column test; the refresh every 32 steps and the row search of a risen
// column (one step late, between the next column's two phases) are the
// only branches.

#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <thread>
#include <vector>

#include "search_internal.cuh"
#include "tpz_common.cuh"

namespace tpz {
namespace sw {

constexpr int kMaxR = 32;           // rows per lane; one stripe = 32 lanes x R rows
constexpr int kStripeRows = 32 * kMaxR;
constexpr int kMaxStripes = (TPZ_SW_MAX_QLEN + kStripeRows - 1) / kStripeRows;
// row bins: b < 32 -> R = b+1, one stripe; b = 32..38 -> R = 32, b-30 stripes
constexpr int kRBins = 40;
constexpr int kSBins = 256;         // subject-length buckets (32 residues each)
constexpr int kBins = kRBins * kSBins;
constexpr int kPadLetter = 25;      // subject column past a pair's end
constexpr int kPadScore = -64;      // profile value of pad rows / pad columns
constexpr int kMatStride = 32;      // shared matrix row stride (bytes)
constexpr int kSmatBytes = 26 * kMatStride;

// profile words per lane and pair: 4 rows per word
__host__ __device__ constexpr int words_for(int R) { return (R + 3) / 4; }
__host__ __device__ constexpr int profile_bytes(int R) { return 26 * 32 * 4 * words_for(R); }
constexpr int kRing = 128;          // subject-letter ring per warp (uint16 letter pairs)
__host__ __device__ constexpr int smem_bytes(int R) {
    return kSmatBytes + 2 * profile_bytes(R) + 2 * kRing;
}
// Fm "cleared" at an SSW lane start: any value <= 0 acts like the cleared
// one there, so the start row adds -kBig instead of masking (exact while
// every score stays below kBig; larger scores take the 32-bit rerun).
constexpr int kBig = 32512;

struct Args {
    const int8_t *q;
    const int64_t *qoff;
    const int32_t *qlen;
    const int8_t *s;
    const int64_t *soff;
    const int32_t *slen;
    int32_t *score, *ref_end, *read_end, *status;
    const int32_t *sorted;   // pair ids sorted by bin
    const int32_t *rinfo;    // per R bin: [start, count]
    int32_t *next_task;      // per R bin task counter
    int32_t *rerun;          // pairs that need the i16 lane length
    int32_t *rerun_count;
    // per row bin (null: one list for all bins): the u8 pass of bin b appends
    // its saturated pairs at rerun + rinfo[2b] and counts them here, so the
    // i16 pass of the bin can follow it on the same stream
    int32_t *rerun_bin_count;
    // null: a bin's pairs are sorted[rinfo[2b] ..] and number rinfo[2b + 1];
    // else the count is task_count[b] (the i16 pass over a bin's rerun list)
    const int32_t *task_count;
    int ssw_lanes;           // 16 (u8 pass) or 8 (i16 pass)
    int gap_open, gap_extend, bias;
    int translate;           // 1: q/s bytes go through xq/xs first
    int score_only;          // 1: scores only, no end coordinates (ref_end = read_end = -2)
    uint32_t *bnd;           // stripe boundary rows, bnd_words per block (multi-stripe bins)
    int64_t bnd_words;
    int32_t *exact_list;     // i16-pass pairs near 32767: re-run in 32-bit arithmetic
    int32_t *exact_count;
    int exact_threshold;
    int8_t mat[625];
    int8_t xq[128], xs[128]; // byte -> matrix index (internal alphabet inputs)
};

__device__ __forceinline__ uint32_t pack2(int lo, int hi) {
    return (uint32_t)(uint16_t)(int16_t)lo | ((uint32_t)(uint16_t)(int16_t)hi << 16);
}
__device__ __forceinline__ int lo16(uint32_t x) { return (int)(int16_t)(x & 0xFFFFu); }
__device__ __forceinline__ int hi16(uint32_t x) { return (int)(int16_t)(x >> 16); }

__device__ __forceinline__ uint64_t best_key(int v, int col, int row) {
    return v > 0 ? ((uint64_t)v << 40) | ((uint64_t)(0xFFFFFF - col) << 16) |
                       (uint64_t)(0xFFFF - row)
                 : 0ull;
}

// letter pair (A low byte, B high byte) of subject column c; past a
// subject's end, and for bytes outside the alphabet, the pad letter
__device__ __forceinline__ uint32_t letter_pair(const Args &a, const int8_t *sA, int slA,
                                                const int8_t *sB, int slB, int c) {
    int la = kPadLetter, lb = kPadLetter;
    if (c < slA) {
        la = sA[c];
        if (a.translate) la = a.xs[la & 127];
        if ((unsigned)la >= 25u) la = kPadLetter;
    }
    if (c < slB) {
        lb = sB[c];
        if (a.translate) lb = a.xs[lb & 127];
        if ((unsigned)lb >= 25u) lb = kPadLetter;
    }
    return (uint32_t)la | ((uint32_t)lb << 8);
}

// One task: pairs pA and pB (pB < 0: none) in the halves of the int16x2
// lanes.  The pass (16 SSW lanes = u8, 8 = i16) comes from `a` (QM = false)
// or, for the query-major kernel, from qm_lanes; saturated u8 results go to
// qm_rerun / qm_rerun_count when given, else to a.rerun / a.rerun_count.
// QM = true also means that profA/profB already hold the query profile
// (both pairs share it).
template <int R, bool MULTI, bool QM = false, bool SCORE = false>
__device__ __forceinline__ void run_task(const Args &a, int pA, int pB, const int8_t *smat,
                                         uint32_t *profA, uint32_t *profB, uint16_t *ring,
                                         int stripes, uint32_t *bnd, int qm_lanes = 0,
                                         int32_t *qm_rerun = nullptr,
                                         int32_t *qm_rerun_count = nullptr) {
    constexpr bool BUILD = !QM;
#define TPZ_LANES (QM ? qm_lanes : a.ssw_lanes)
    constexpr int W = words_for(R);
    const int lane = threadIdx.x & 31;

    const int qlA = a.qlen[pA];
    const int slA = a.slen[pA];
    const int8_t *qA = a.q + a.qoff[pA];
    const int8_t *sA = a.s + a.soff[pA];
    const int qlB = pB >= 0 ? a.qlen[pB] : 0;
    const int slB = pB >= 0 ? a.slen[pB] : 0;
    const int8_t *qB = pB >= 0 ? a.q + a.qoff[pB] : qA;
    const int8_t *sB = pB >= 0 ? a.s + a.soff[pB] : sA;
    const int N = max(slA, slB);
    const int segA = max(1, (qlA + TPZ_LANES - 1) / TPZ_LANES);
    const int segB = max(1, (qlB + TPZ_LANES - 1) / TPZ_LANES);
    const uint32_t NGO = pack2(-a.gap_open, -a.gap_open);
    const uint32_t NGE = pack2(-a.gap_extend, -a.gap_extend);
    const uint32_t NEGINF = 0x80008000u;
    // sign-extend byte r%4 of the A word into the low half, of the B word
    // into the high half
    constexpr uint32_t SEL[4] = {0xC480u, 0xD591u, 0xE6A2u, 0xF7B3u};
    uint64_t kA = 0, kB = 0;
    bool decided = false;      // u8 pass: both pairs already go to the i16 pass

    // Queries longer than one stripe (32 lanes x R rows) run stripe after
    // stripe; the last row of a stripe (H, F, Fm per column) goes to `bnd`
    // and enters the next stripe at lane 0.  Lane 0 reads column k at step k
    // and lane 31 writes column k-31 at step k, so one buffer serves as both.
    const int nstripes = MULTI ? stripes : 1;
    for (int st = 0; st < nstripes; ++st) {
    const int i0 = (st * 32 + lane) * R;

    // ---- profile of this lane's rows for all 26 letters (25 + pad column),
    // word w of letter l at [(l * W + w) * 32 + lane]: conflict-free per lane
    if constexpr (BUILD) {
    int qa[R], qb[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        qa[r] = (i0 + r < qlA) ? qA[i0 + r] : -1;
        qb[r] = (i0 + r < qlB) ? qB[i0 + r] : -1;
        if (a.translate) {
            if (qa[r] >= 0) qa[r] = a.xq[qa[r] & 127];
            if (qb[r] >= 0) qb[r] = a.xq[qb[r] & 127];
        }
        if (qa[r] >= 25) qa[r] = -1;
        if (qb[r] >= 25) qb[r] = -1;
    }
    __syncwarp();
    for (int let = 0; let < 26; ++let) {
        const int8_t *mrow = smat + let * kMatStride;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            uint32_t wa = 0, wb = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int r = 4 * w + k;
                int va = kPadScore, vb = kPadScore;
                if (r < R) {
                    if (qa[r] >= 0) va = mrow[qa[r]];
                    if (qb[r] >= 0) vb = mrow[qb[r]];
                }
                wa |= (uint32_t)(uint8_t)(int8_t)va << (8 * k);
                wb |= (uint32_t)(uint8_t)(int8_t)vb << (8 * k);
            }
            profA[(let * W + w) * 32 + lane] = wa;
            profB[(let * W + w) * 32 + lane] = wb;
        }
    }
    }   // BUILD
    // ---- subject letters: columns 0..63 in the ring, 64..95 in flight;
    // every 32 steps the lanes store the next 32 columns and fetch 32 more
    ring[lane] = (uint16_t)letter_pair(a, sA, slA, sB, slB, lane);
    ring[32 + lane] = (uint16_t)letter_pair(a, sA, slA, sB, slB, 32 + lane);
    ring[64 + lane] = (uint16_t)(kPadLetter | (kPadLetter << 8));
    ring[96 + lane] = (uint16_t)(kPadLetter | (kPadLetter << 8));
    uint32_t pre = letter_pair(a, sA, slA, sB, slB, 64 + lane);
    __syncwarp();

    // ---- SSW lane starts: the Fm terms of a start row add -kBig
    uint32_t ngo[R], nge[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const bool sa = (i0 + r) % segA == 0, sb = (i0 + r) % segB == 0;
        ngo[r] = pack2(sa ? -kBig : -a.gap_open, sb ? -kBig : -a.gap_open);
        nge[r] = pack2(sa ? -kBig : -a.gap_extend, sb ? -kBig : -a.gap_extend);
    }

    uint32_t E[R], H[R];
#pragma unroll
    for (int r = 0; r < R; ++r) { E[r] = 0u; H[r] = 0u; }

    uint32_t outH = 0u, outF = 0u, outFm = 0u;
    uint32_t diag = 0u;
    uint32_t runmax = 0u, wmax = 0u;
    int colA = -1, rowA = 0, colB = -1, rowB = 0;

    // profile words of this step's column (j = k - lane), fetched one step
    // ahead; the letter pair of the column after it
    uint32_t wa[W], wb[W];
    {
        const uint32_t l = ring[(-lane) & (kRing - 1)];
#pragma unroll
        for (int w = 0; w < W; ++w) {
            wa[w] = profA[((l & 0xFFu) * W + w) * 32 + lane];
            wb[w] = profB[((l >> 8) * W + w) * 32 + lane];
        }
    }
    uint32_t let1 = ring[(1 - lane) & (kRing - 1)];

    // The row search of a column whose maximum rose runs one step late,
    // between the next column's diagonal terms and its F / Fm chains: H still
    // holds the risen column there, and the vote that guards the search then
    // waits on nothing, so no step stalls on the one before it.
    bool pend = false;                   // the previous column needs its row found
    uint32_t pcm = 0u, pthr = 0u;        // its column maximum and threshold
    int pj = 0;                          // its column
    auto search = [&]() {
        if (!a.score_only && __any_sync(0xFFFFFFFFu, pend)) {
            // smallest row holding the column maximum, both halves at once:
            // max(H - cm, -1) is 0 on rows holding it and -1 elsewhere; those
            // rows contribute R - r and the largest contribution wins
            const uint32_t negv = __viaddmax_s16x2(~pcm, 0x00010001u, NEGINF);
            uint32_t acc = 0u;
#pragma unroll
            for (int r = 0; r < R; r += 2) {
                const uint32_t g0 =
                    ~__viaddmax_s16x2(H[r], negv, 0xFFFFFFFFu) & pack2(R - r, R - r);
                if (r + 1 < R) {
                    const uint32_t g1 = ~__viaddmax_s16x2(H[r + 1], negv, 0xFFFFFFFFu) &
                                        pack2(R - r - 1, R - r - 1);
                    acc = __vimax3_s16x2(acc, g0, g1);
                } else {
                    acc = __vimax_s16x2_relu(acc, g0);
                }
            }
            if (pend) {
                if (lo16(pcm) > lo16(pthr)) { colA = pj; rowA = i0 + R - lo16(acc); }
                if (hi16(pcm) > hi16(pthr)) { colB = pj; rowB = i0 + R - hi16(acc); }
            }
        }
        pend = false;
    };

    auto step = [&](const int k, const uint32_t (&cwa)[W], const uint32_t (&cwb)[W],
                    uint32_t (&nwa)[W], uint32_t (&nwb)[W]) {
        const int j = k - lane;
        uint32_t inH = __shfl_up_sync(0xFFFFFFFFu, outH, 1);
        uint32_t inF = __shfl_up_sync(0xFFFFFFFFu, outF, 1);
        uint32_t inFm = __shfl_up_sync(0xFFFFFFFFu, outFm, 1);
        if (lane == 0) {
            if (MULTI && st > 0 && k < N) {
                const uint32_t *b = bnd + 3 * (size_t)k;
                inH = b[0]; inF = b[1]; inFm = b[2];
            } else {
                inH = 0u; inF = 0u; inFm = 0u;
            }
        }
        // next step's profile words
#pragma unroll
        for (int w = 0; w < W; ++w) {
            nwa[w] = profA[((let1 & 0xFFu) * W + w) * 32 + lane];
            nwb[w] = profB[((let1 >> 8) * W + w) * 32 + lane];
        }
        let1 = ring[(j + 2) & (kRing - 1)];
        // every lane computes every step: a lane before its first column
        // (j < 0) sees pad letters and zero inputs, so its H stays 0 and its
        // E only goes negative, which no later cell can see through the
        // relu; past the subject's end (j >= N) the pad columns only hold
        // values below a real cell's, which can never be the maximum
        uint32_t F = inF, Fm = inFm, D = diag;
        // first every row's diagonal term and its gap-open candidate (they
        // depend only on the previous column), then the F / Fm chains, the
        // only row-to-row dependences, with E and H hanging off them
        uint32_t Xa[R], Xga[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t sc = prmt(cwa[r >> 2], cwb[r >> 2], SEL[r & 3]);
            Xa[r] = __viaddmax_s16x2_relu(r == 0 ? D : H[r - 1], sc, E[r]);
            Xga[r] = __viaddmax_s16x2(Xa[r], NGO, NEGINF);
        }
        if constexpr (!SCORE) search();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t Hn = __vimax_s16x2_relu(Xa[r], F);
            const uint32_t Gp = __viaddmax_s16x2(Fm, ngo[r], Xga[r]);
            E[r] = __viaddmax_s16x2(E[r], NGE, Gp);
            F = __viaddmax_s16x2(F, NGE, Xga[r]);
            Fm = __viaddmax_s16x2(Fm, nge[r], Xga[r]);
            H[r] = Hn;
        }
        // column maximum of the lane's rows, floored at the search threshold
        // max(running max, warp maximum - 1): a half needs its row found when
        // it rises above the threshold, i.e. above the lane's running max and
        // not below the warp maximum of the last refresh (anything lower
        // cannot be the alignment maximum).  The running max may so take the
        // value warp maximum - 1 without a cell holding it; such a lane can
        // never hold the final maximum.
        const uint32_t thr = __viaddmax_s16x2(wmax, 0xFFFFFFFFu, runmax);
        uint32_t cm = thr;
#pragma unroll
        for (int r = 0; r + 1 < R; r += 2) cm = __vimax3_s16x2(cm, H[r], H[r + 1]);
        if (R & 1) cm = __vimax_s16x2_relu(cm, H[R - 1]);
        outH = H[R - 1];
        outF = F;
        outFm = Fm;
        if (MULTI && lane == 31 && st + 1 < stripes && j >= 0 && j < N) {
            uint32_t *b = bnd + 3 * (size_t)j;
            b[0] = outH; b[1] = outF; b[2] = outFm;
        }
        if constexpr (!SCORE) {
            pend = cm != thr;
            pcm = cm;
            pthr = thr;
            pj = j;
        }
        runmax = cm;
        diag = inH;
    };
    uint32_t wa2[W], wb2[W];
    // an even step count; a step past N + 30 finds every lane past the end
    const int steps = (N + 32) & ~1;
    for (int k0 = 0; k0 < steps; k0 += 32) {
        if (k0 > 0) {
            // every 32 steps the lanes store the next 32 columns' letters and
            // fetch 32 more
            ring[(k0 + 32 + lane) & (kRing - 1)] = (uint16_t)pre;
            pre = letter_pair(a, sA, slA, sB, slB, k0 + 64 + lane);
            // warp maximum so far: a lane's rise below it cannot end up as
            // the alignment's maximum, so it needs no row search
            uint32_t wm = runmax;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                wm = __vimax_s16x2_relu(wm, __shfl_xor_sync(0xFFFFFFFFu, wm, o));
            if (TPZ_LANES == 16) {
                // u8 pass: a pair whose maximum reached 255 - bias is decided
                // (the i16 pass reruns it), so it needs no more row searches,
                // and a task whose pairs are both decided stops here
                const bool da = lo16(wm) + a.bias >= 255, db = hi16(wm) + a.bias >= 255;
                if (da) wm = (wm & 0xFFFF0000u) | 0x7FFFu;
                if (db) wm = (wm & 0x0000FFFFu) | 0x7FFF0000u;
                if (da && (db || pB < 0)) decided = true;
            }
            wmax = wm;
            __syncwarp();
            if (decided) break;
        }
        const int kend = min(k0 + 32, steps);
        for (int k = k0; k < kend; k += 2) {
            step(k, wa, wb, wa2, wb2);
            step(k + 1, wa2, wb2, wa, wb);
        }
    }
    if constexpr (!SCORE) search();     // the last column's, if it rose

    if (a.score_only || decided) { colA = colB = 0; rowA = rowB = 0; }
    kA = max(kA, best_key(lo16(runmax), colA, rowA));
    kB = max(kB, best_key(hi16(runmax), colB, rowB));
    __syncwarp();
    if (decided) break;
    }   // stripes

    // ---- warp reduction: max value, then first column, then smallest row
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kA = max(kA, __shfl_xor_sync(0xFFFFFFFFu, kA, o));
        kB = max(kB, __shfl_xor_sync(0xFFFFFFFFu, kB, o));
    }
    if (lane < 2) {
        const int p = lane == 0 ? pA : pB;
        const uint64_t key = lane == 0 ? kA : kB;
        if (p >= 0) {
            const int v = (int)(key >> 40);
            const int col = key ? 0xFFFFFF - (int)((key >> 16) & 0xFFFFFF) : -1;
            const int row = key ? 0xFFFF - (int)(key & 0xFFFF) : 0;
            if (TPZ_LANES == 16 && v + a.bias >= 255) {
                // u8 pass saturated: the i16 pass decides (src/ssw.c:863-865)
                int32_t *rr = qm_rerun ? qm_rerun : a.rerun;
                const int slot = atomicAdd(qm_rerun ? qm_rerun_count : a.rerun_count, 1);
                rr[slot] = p;
            } else if (TPZ_LANES == 8 && a.exact_list && v >= a.exact_threshold) {
                // near the i16 limit: 16-bit lanes may wrap, redo in 32 bits
                const int slot = atomicAdd(a.exact_count, 1);
                a.exact_list[slot] = p;
            } else {
                a.score[p] = v;
                a.ref_end[p] = a.score_only ? -2 : col;
                a.read_end[p] = a.score_only ? -2 : row;
                a.status[p] = TPZ_SW_OK;
            }
        }
    }
}

#undef TPZ_LANES

template <int R>
__global__ void __launch_bounds__(32) sw_bin_kernel(const __grid_constant__ Args a, int bin,
                                                    int stripes) {
    extern __shared__ __align__(16) uint8_t smem[];
    int8_t *smat = reinterpret_cast<int8_t *>(smem);
    uint32_t *profA = reinterpret_cast<uint32_t *>(smem + kSmatBytes);
    uint32_t *profB = profA + profile_bytes(R) / 4;
    uint16_t *ring = reinterpret_cast<uint16_t *>(profB + profile_bytes(R) / 4);
    const int lane = threadIdx.x;
    const int start = a.rinfo[2 * bin];
    const int count = a.task_count ? a.task_count[bin] : a.rinfo[2 * bin + 1];
    const int ntask = (count + 1) / 2;
    if (ntask == 0) return;
    int32_t *rr_list = a.rerun_bin_count ? a.rerun + start : nullptr;
    int32_t *rr_count = a.rerun_bin_count ? a.rerun_bin_count + bin : nullptr;

    for (int i = lane; i < 26 * kMatStride; i += 32) {
        const int r = i / kMatStride, c = i % kMatStride;
        smat[i] = (r < 25 && c < 25) ? a.mat[r * 25 + c] : (int8_t)kPadScore;
    }
    __syncwarp();
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(&a.next_task[bin], 1);
        t = __shfl_sync(0xFFFFFFFFu, t, 0);
        if (t >= ntask) break;
        const int pA = a.sorted[start + 2 * t];
        const int pB = 2 * t + 1 < count ? a.sorted[start + 2 * t + 1] : -1;
        if constexpr (R == kMaxR) {
            if (stripes > 1) {
                run_task<R, true>(a, pA, pB, smat, profA, profB, ring, stripes,
                                  a.bnd + (size_t)blockIdx.x * a.bnd_words, 0, rr_list,
                                  rr_count);
                continue;
            }
        }
        run_task<R, false>(a, pA, pB, smat, profA, profB, ring, 1, nullptr, 0, rr_list, rr_count);
    }
}

// One pair per launch (the per-pair form of ssw_init + ssw_align): the u8
// lane pass and, when it saturates, the i16 lane pass in the same launch.
// Pair lengths and the rerun flag live in shared memory.
template <int R>
__global__ void __launch_bounds__(32) sw_one_kernel(const __grid_constant__ Args a, int qlen,
                                                    int slen) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ int64_t s_off;
    __shared__ int32_t s_ql, s_sl, s_rr[2];
    int8_t *smat = reinterpret_cast<int8_t *>(smem);
    uint32_t *profA = reinterpret_cast<uint32_t *>(smem + kSmatBytes);
    uint32_t *profB = profA + profile_bytes(R) / 4;
    uint16_t *ring = reinterpret_cast<uint16_t *>(profB + profile_bytes(R) / 4);
    const int lane = threadIdx.x;
    for (int i = lane; i < 26 * kMatStride; i += 32) {
        const int r = i / kMatStride, c = i % kMatStride;
        smat[i] = (r < 25 && c < 25) ? a.mat[r * 25 + c] : (int8_t)kPadScore;
    }
    if (lane == 0) { s_off = 0; s_ql = qlen; s_sl = slen; s_rr[0] = 0; s_rr[1] = 0; }
    __syncwarp();
    Args b = a;
    b.qoff = &s_off; b.soff = &s_off; b.qlen = &s_ql; b.slen = &s_sl;
    b.rerun_count = &s_rr[0]; b.rerun = &s_rr[1];
    b.ssw_lanes = 16;
    run_task<R, false>(b, 0, -1, smat, profA, profB, ring, 1, nullptr);
    __syncwarp();
    if (s_rr[0]) {
        // the u8 pass saturated: the i16 pass decides (src/ssw.c:863-865)
        b.ssw_lanes = 8;
        run_task<R, false>(b, 0, -1, smat, profA, profB, ring, 1, nullptr);
    }
}

// ------------------------------------------------------------- query-major

// Pairs that share their query (the hits of one search query): a block of
// kQmWarps warps per query keeps ONE profile of the query in shared memory
// for all of them, so a warp costs the SM a fraction of the shared memory
// of the pair-per-task kernel and more warps hide the DPX latency.  The
// block sorts the query's pairs by subject length (longest first, two per
// task), runs the u8 pass over all of them and then, with the profile
// still resident, the i16 pass over those that saturated.
constexpr int kQmWarps = 8;
constexpr int kQmMaxPairs = 256;      // pairs per chunk: longer pair lists of a query are cut
constexpr int kQmMinPairs = 2 * kQmWarps;
constexpr int kQmStreams = 8;

__host__ __device__ constexpr int qm_smem_bytes(int R) {
    return kSmatBytes + profile_bytes(R) + kQmWarps * 2 * kRing + 8 * kQmMaxPairs +
           4 * kQmMaxPairs;
}

struct QmArgs {
    const int64_t *chunks;    // [first pair, end) per chunk; the pairs of a chunk share the query
    const int32_t *bin_info;  // per row bin R-1: [first chunk, count]
    int32_t *next;            // per row bin: chunk counter
};

// profile words of letters warp, warp + kQmWarps, ... for lane's rows of the
// query of pair p
template <int R>
__device__ __forceinline__ void qm_build_profile(const Args &a, int64_t p, const int8_t *smat,
                                                 uint32_t *prof, int warp, int lane) {
    constexpr int W = words_for(R);
    const int ql = a.qlen[p];
    const int8_t *qp = a.q + a.qoff[p];
    const int i0 = lane * R;
    int qv[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        int x = (i0 + r < ql) ? qp[i0 + r] : -1;
        if (a.translate && x >= 0) x = a.xq[x & 127];
        qv[r] = (x >= 25) ? -1 : x;
    }
    for (int let = warp; let < 26; let += kQmWarps) {
        const int8_t *mrow = smat + let * kMatStride;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            uint32_t word = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int r = 4 * w + k;
                int v = kPadScore;
                if (r < R && qv[r] >= 0) v = mrow[qv[r]];
                word |= (uint32_t)(uint8_t)(int8_t)v << (8 * k);
            }
            prof[(let * W + w) * 32 + lane] = word;
        }
    }
}

// SCORE: scores only (report-mode search), with the end-coordinate row
// search compiled out rather than skipped at run time
template <int R, bool SCORE>
__global__ void __launch_bounds__(kQmWarps * 32) sw_query_kernel(const __grid_constant__ Args a,
                                                                 QmArgs g, int bin) {
    extern __shared__ __align__(16) uint8_t smem[];
    int8_t *smat = reinterpret_cast<int8_t *>(smem);
    uint32_t *prof = reinterpret_cast<uint32_t *>(smem + kSmatBytes);
    uint16_t *rings = reinterpret_cast<uint16_t *>(prof + profile_bytes(R) / 4);
    uint64_t *keys = reinterpret_cast<uint64_t *>(rings + kQmWarps * kRing);
    int32_t *sat = reinterpret_cast<int32_t *>(keys + kQmMaxPairs);
    __shared__ int s_group, s_next, s_nsat;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint16_t *ring = rings + warp * kRing;
    const int gb = g.bin_info[2 * bin], gc = g.bin_info[2 * bin + 1];
    if (gc == 0) return;
    for (int i = threadIdx.x; i < 26 * kMatStride; i += blockDim.x) {
        const int r = i / kMatStride, c = i % kMatStride;
        smat[i] = (r < 25 && c < 25) ? a.mat[r * 25 + c] : (int8_t)kPadScore;
    }
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            s_group = atomicAdd(&g.next[bin], 1);
            s_next = 0;
            s_nsat = 0;
        }
        __syncthreads();
        if (s_group >= gc) break;
        const int64_t p0 = g.chunks[2 * (gb + s_group)];
        const int n = (int)(g.chunks[2 * (gb + s_group) + 1] - p0);
        int np = 1;
        while (np < n) np <<= 1;
        // keys: subject length + 1 (descending), pair id; padding 0 sorts last
        for (int i = threadIdx.x; i < np; i += blockDim.x)
            keys[i] = i < n ? ((uint64_t)(uint32_t)(a.slen[p0 + i] + 1) << 32) | (uint32_t)(p0 + i)
                            : 0ull;
        qm_build_profile<R>(a, p0, smat, prof, warp, lane);
        __syncthreads();
        for (int k = 2; k <= np; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < np; i += blockDim.x) {
                    const int l = i ^ j;
                    if (l > i) {
                        const uint64_t x = keys[i], y = keys[l];
                        if (((i & k) == 0) ? (x < y) : (x > y)) { keys[i] = y; keys[l] = x; }
                    }
                }
                __syncthreads();
            }
        }
        // u8 pass over every pair of the query
        for (;;) {
            int t = 0;
            if (lane == 0) t = atomicAdd(&s_next, 1);
            t = __shfl_sync(0xFFFFFFFFu, t, 0);
            if (2 * t >= n) break;
            const int pA = (int)(uint32_t)keys[2 * t];
            const int pB = 2 * t + 1 < n ? (int)(uint32_t)keys[2 * t + 1] : -1;
            run_task<R, false, true, SCORE>(a, pA, pB, smat, prof, prof, ring, 1, nullptr, 16, sat,
                                     &s_nsat);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_next = 0;
        __syncthreads();
        // i16 pass over the pairs that saturated (src/ssw.c:863-865)
        const int ns = s_nsat;
        for (;;) {
            int t = 0;
            if (lane == 0) t = atomicAdd(&s_next, 1);
            t = __shfl_sync(0xFFFFFFFFu, t, 0);
            if (2 * t >= ns) break;
            const int pA = sat[2 * t];
            const int pB = 2 * t + 1 < ns ? sat[2 * t + 1] : -1;
            run_task<R, false, true, SCORE>(a, pA, pB, smat, prof, prof, ring, 1, nullptr, 8, nullptr,
                                     nullptr);
        }
    }
}

// ---------------------------------------------------------------- binning

__device__ __forceinline__ int pair_bin(int ql, int sl) {
    const int rb = ql <= kStripeRows ? (ql + 31) / 32 - 1                 // 0..31
                                     : 30 + (ql + kStripeRows - 1) / kStripeRows;  // 32..38
    const int sb = min(sl >> 5, kSBins - 1);
    return rb * kSBins + (kSBins - 1 - sb);             // long subjects first
}

// list == nullptr: pairs 0..n-1; else list[0 .. *list_n)
__global__ void bin_count_kernel(int64_t n, const int32_t *list, const int32_t *list_n,
                                 const int32_t *qlen, const int32_t *slen, int32_t *counts,
                                 int32_t *status, int max_qlen, int32_t *multi_maxn) {
    const int64_t limit = list ? (int64_t)*list_n : n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int p = list ? list[i] : (int)i;
        const int ql = qlen[p], sl = slen[p];
        if (ql < 1 || ql > max_qlen || sl < 0 || sl >= TPZ_SW_MAX_SLEN) {
            status[p] = TPZ_SW_INVALID;
            continue;
        }
        atomicAdd(&counts[pair_bin(ql, sl)], 1);
        if (ql > kStripeRows && multi_maxn) atomicMax(multi_maxn, sl);
    }
}

__global__ void set_i32_kernel(int32_t *p, int32_t v) { *p = v; }

// one block of 1024 threads: exclusive scan of kBins counts -> cursor; the
// per-R-bin [start, count] pairs -> rinfo; task counters cleared.
__global__ void bin_scan_kernel(const int32_t *counts, int32_t *cursor, int32_t *rinfo,
                                int32_t *next_task) {
    constexpr int PER = kBins / 1024;
    __shared__ int32_t part[1024];
    const int t = threadIdx.x;
    int32_t loc[PER];
    int32_t sum = 0;
#pragma unroll
    for (int i = 0; i < PER; ++i) { loc[i] = counts[t * PER + i]; sum += loc[i]; }
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int32_t v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int32_t run = part[t] - sum;
#pragma unroll
    for (int i = 0; i < PER; ++i) { cursor[t * PER + i] = run; run += loc[i]; }
    __syncthreads();
    if (t < kRBins) {
        const int b0 = t * kSBins, b1 = b0 + kSBins;
        const int32_t s0 = cursor[b0];
        const int32_t e1 = cursor[b1 - 1] + counts[b1 - 1];
        rinfo[2 * t] = s0;
        rinfo[2 * t + 1] = e1 - s0;
        next_task[t] = 0;
    }
}

__global__ void bin_scatter_kernel(int64_t n, const int32_t *list, const int32_t *list_n,
                                   const int32_t *qlen, const int32_t *slen, int32_t *cursor,
                                   int32_t *sorted, int max_qlen) {
    const int64_t limit = list ? (int64_t)*list_n : n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int p = list ? list[i] : (int)i;
        const int ql = qlen[p], sl = slen[p];
        if (ql < 1 || ql > max_qlen || sl < 0 || sl >= TPZ_SW_MAX_SLEN) continue;
        const int pos = atomicAdd(&cursor[pair_bin(ql, sl)], 1);
        sorted[pos] = p;
    }
}

// ------------------------------------------------------------ roofline probe

// Independent chains of __viaddmax_s16x2 per thread: measures the DPX issue
// rate the SW kernel is bounded by.  kChains chains per thread, iters steps.
constexpr int kProbeChains = 8;

__global__ void __launch_bounds__(256) dpx_probe_kernel(int iters, uint32_t inc, uint32_t floor_v,
                                                        uint32_t *out) {
    uint32_t acc[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) acc[c] = (threadIdx.x + 131u * c) * 0x00010001u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c) acc[c] = __viaddmax_s16x2(acc[c], inc, floor_v);
    }
    uint32_t x = 0;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) x ^= acc[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

// ------------------------------------------------------------ host driver

typedef void (*KernelFn)(const Args, int, int);

template <int R>
struct Table {
    static void fill(KernelFn *k) {
        k[R - 1] = sw_bin_kernel<R>;
        Table<R - 1>::fill(k);
    }
};
template <>
struct Table<0> {
    static void fill(KernelFn *) {}
};

constexpr int kAuxStreams = 8;

struct LaunchCfg {
    KernelFn fn[kMaxR];
    int smem[kMaxR];
    int blocks_per_sm[kMaxR];
    cudaStream_t aux[kAuxStreams];       // bin kernels overlap their tails here
    cudaEvent_t fork, join[kAuxStreams];
    int32_t *maxn_pin;                   // pinned copy of a call's multi-stripe maximum
    cudaEvent_t maxn_ready;
};

// Per host thread and device: the auxiliary streams and fork/join events of
// one call must not be shared with a call running in another thread.
struct LaunchCfgs {
    std::vector<LaunchCfg *> per_dev;
    ~LaunchCfgs() {
        for (LaunchCfg *c : per_dev) {
            if (!c) continue;
            for (int i = 0; i < kAuxStreams; ++i) {
                cudaStreamDestroy(c->aux[i]);
                cudaEventDestroy(c->join[i]);
            }
            cudaEventDestroy(c->fork);
            cudaEventDestroy(c->maxn_ready);
            cudaFreeHost(c->maxn_pin);
            delete c;
        }
    }
};

// lane: calls of one thread that run at the same time (the chunks of the
// host entry point) take different lanes, so they get separate streams
static int launch_cfg(const LaunchCfg **out, int lane = 0) {
    static thread_local LaunchCfgs cfgs;
    std::vector<LaunchCfg *> &per_dev = cfgs.per_dev;
    int dev = 0;
    TPZ_CUDA(cudaGetDevice(&dev));
    dev = 2 * dev + (lane & 1);
    if ((int)per_dev.size() <= dev) per_dev.resize(dev + 1, nullptr);
    if (!per_dev[dev]) {
        LaunchCfg *c = new LaunchCfg();
        Table<kMaxR>::fill(c->fn);
        for (int r = 1; r <= kMaxR; ++r) {
            c->smem[r - 1] = smem_bytes(r);
            TPZ_CUDA(cudaFuncSetAttribute((const void *)c->fn[r - 1],
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          c->smem[r - 1]));
            // one carveout for every bin kernel, so blocks of concurrently
            // running bins can share an SM
            TPZ_CUDA(cudaFuncSetAttribute((const void *)c->fn[r - 1],
                                          cudaFuncAttributePreferredSharedMemoryCarveout,
                                          (int)cudaSharedmemCarveoutMaxShared));
            int nb = 0;
            TPZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void *)c->fn[r - 1],
                                                                   32, c->smem[r - 1]));
            c->blocks_per_sm[r - 1] = std::max(1, nb);
        }
        for (int i = 0; i < kAuxStreams; ++i) {
            TPZ_CUDA(cudaStreamCreateWithFlags(&c->aux[i], cudaStreamNonBlocking));
            TPZ_CUDA(cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming));
        }
        TPZ_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
        TPZ_CUDA(cudaEventCreateWithFlags(&c->maxn_ready, cudaEventDisableTiming));
        TPZ_CUDA(cudaHostAlloc((void **)&c->maxn_pin, sizeof(int32_t), cudaHostAllocDefault));
        per_dev[dev] = c;
    }
    *out = per_dev[dev];
    return TPZ_OK;
}

static thread_local int64_t g_last_launches = 0;

// R and stripe count of a row bin
__host__ __device__ constexpr int bin_rows(int b) { return b < kMaxR ? b + 1 : kMaxR; }
__host__ __device__ constexpr int bin_stripes(int b) { return b < kMaxR ? 1 : b - 30; }
constexpr int kUsedRBins = kMaxR + kMaxStripes - 1;     // 39

// One pass over the pairs (all of them, or list[0 .. *list_n)): counting sort
// into row bins, then one persistent kernel per bin.  With a16, each bin's
// kernel is followed on its stream by the i16 pass over the pairs of that bin
// that saturated, so no pass waits for the whole batch.
static int launch_round(const LaunchCfg *cfg, Args &a, int64_t n, const int32_t *list,
                        const int32_t *list_n, int32_t *counts, int32_t *cursor, int32_t *sorted,
                        int32_t *multi_maxn, cudaStream_t st, int64_t &launches,
                        int *host_maxn, int known_maxn = -1, Args *a16 = nullptr) {
    const int nsm = sm_count();
    TPZ_CUDA(cudaMemsetAsync(counts, 0, sizeof(int32_t) * kBins, st));
    const int gb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)nsm * 8);
    bin_count_kernel<<<std::max(gb, 1), 256, 0, st>>>(n, list, list_n, a.qlen, a.slen, counts,
                                                      a.status, TPZ_SW_MAX_QLEN, multi_maxn);
    bin_scan_kernel<<<1, 1024, 0, st>>>(counts, cursor, const_cast<int32_t *>(a.rinfo),
                                        a.next_task);
    bin_scatter_kernel<<<std::max(gb, 1), 256, 0, st>>>(n, list, list_n, a.qlen, a.slen, cursor,
                                                        sorted, TPZ_SW_MAX_QLEN);
    launches += 4;
    // The boundary buffer of multi-stripe bins is sized by the longest subject
    // among queries longer than one stripe.  When the caller does not know it,
    // the device's count comes back while the single-stripe bins already run,
    // and the multi-stripe bins are launched after them.
    const bool defer = host_maxn && known_maxn < 0;
    auto alloc_bnd = [&](int maxn, cudaStream_t s) -> int {
        a.bnd_words = 3 * ((int64_t)maxn + 1);
        const size_t bytes = sizeof(uint32_t) * (size_t)a.bnd_words * nsm *
                             cfg->blocks_per_sm[kMaxR - 1];
        TPZ_CUDA(cudaMallocAsync((void **)&a.bnd, bytes, s));
        if (a16) { a16->bnd = a.bnd; a16->bnd_words = a.bnd_words; }
        return TPZ_OK;
    };
    if (host_maxn && !defer) {
        *host_maxn = known_maxn;
        if (known_maxn > 0) {
            const int rc = alloc_bnd(known_maxn, st);
            if (rc) return rc;
        }
    }
    if (defer) {
        TPZ_CUDA(cudaMemcpyAsync(cfg->maxn_pin, multi_maxn, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        TPZ_CUDA(cudaEventRecord(cfg->maxn_ready, st));
    }
    // one persistent kernel per row bin, longest rows first, spread over the
    // auxiliary streams so that each kernel's tail overlaps the next one;
    // the multi-stripe bins share one boundary buffer and stay on aux[0]
    TPZ_CUDA(cudaEventRecord(cfg->fork, st));
    for (int i = 0; i < kAuxStreams; ++i) TPZ_CUDA(cudaStreamWaitEvent(cfg->aux[i], cfg->fork, 0));
    int rr = 0;
    auto launch_bin = [&](int b) {
        const int R = bin_rows(b), S = bin_stripes(b);
        const int grid = nsm * cfg->blocks_per_sm[R - 1];
        cudaStream_t xs = S > 1 ? cfg->aux[0] : cfg->aux[rr++ % kAuxStreams];
        cfg->fn[R - 1]<<<grid, 32, cfg->smem[R - 1], xs>>>(a, b, S);
        ++launches;
        if (a16) {
            cfg->fn[R - 1]<<<grid, 32, cfg->smem[R - 1], xs>>>(*a16, b, S);
            ++launches;
        }
    };
    for (int b = kUsedRBins - 1; b >= 0; --b) {
        if (bin_stripes(b) > 1 && (defer || !a.bnd)) continue;
        launch_bin(b);
    }
    int rc = TPZ_OK;
    if (defer) {
        const cudaError_t e = cudaEventSynchronize(cfg->maxn_ready);
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "multi-stripe maximum");
        } else {
            *host_maxn = *cfg->maxn_pin;
            if (*host_maxn > 0 && (rc = alloc_bnd(*host_maxn, cfg->aux[0])) == TPZ_OK)
                for (int b = kUsedRBins - 1; b >= kMaxR; --b) launch_bin(b);
        }
    }
    // the join comes after every launch, also on an error above, so that the
    // caller's stream waits for all kernels before it frees their buffers
    for (int i = 0; i < kAuxStreams; ++i) {
        TPZ_CUDA(cudaEventRecord(cfg->join[i], cfg->aux[i]));
        TPZ_CUDA(cudaStreamWaitEvent(st, cfg->join[i], 0));
    }
    if (rc) return rc;
    TPZ_CUDA(cudaGetLastError());
    return TPZ_OK;
}

// 32-bit re-run of i16-pass pairs whose maximum came near 32767 (16-bit
// lanes could wrap there): the same recurrence with the i16 lane length,
// one thread per pair, rows and columns in a plain loop.  Only pairs whose
// score can pass 32767 - 2*max(M) get here -- query and subject both longer
// than ~1900 residues of near-identity.
constexpr int kExactThreads = 128;

__global__ void __launch_bounds__(kExactThreads) sw_exact_kernel(const __grid_constant__ Args a,
                                                                 int32_t *scratch) {
    const int n = *a.exact_count;
    int32_t *E = scratch + (size_t)threadIdx.x * 2 * TPZ_SW_MAX_QLEN;
    int32_t *Hc = E + TPZ_SW_MAX_QLEN;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int p = a.exact_list[i];
        const int ql = a.qlen[p], sl = a.slen[p];
        const int8_t *qp = a.q + a.qoff[p];
        const int8_t *sp = a.s + a.soff[p];
        const int seg = max(1, (ql + 7) / 8);
        for (int r = 0; r < ql; ++r) { E[r] = 0; Hc[r] = 0; }
        int best = 0, bc = -1, br = 0;
        for (int c = 0; c < sl; ++c) {
            int sc = sp[c];
            if (a.translate) sc = a.xs[sc & 127];
            const int8_t *mrow = a.mat + 25 * sc;
            int F = 0, Fm = 0, D = 0;
            for (int r = 0; r < ql; ++r) {
                if (r % seg == 0) Fm = 0;
                int qc = qp[r];
                if (a.translate) qc = a.xq[qc & 127];
                const int X = max(max(0, D + mrow[qc]), E[r]);
                const int h = max(X, F);
                const int Xg = X - a.gap_open;
                const int Gp = max(Fm - a.gap_open, Xg);
                E[r] = max(E[r] - a.gap_extend, Gp);
                F = max(F - a.gap_extend, Xg);
                Fm = max(Fm - a.gap_extend, Xg);
                D = Hc[r];
                Hc[r] = h;
                if (h > best) { best = h; bc = c; br = r; }
            }
        }
        if (best >= 32767) {
            a.score[p] = 32767; a.ref_end[p] = -1; a.read_end[p] = -1; a.status[p] = TPZ_SW_DROPPED;
        } else {
            a.score[p] = best; a.ref_end[p] = bc; a.read_end[p] = best > 0 ? br : 0;
            a.status[p] = TPZ_SW_OK;
        }
    }
}

int batch_device_x(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                   const int8_t *s, const int64_t *soff, const int32_t *slen, const int8_t *mat,
                   int go, int ge, int32_t *score, int32_t *ref_end, int32_t *read_end,
                   int32_t *status, cudaStream_t st, const int8_t *xq, const int8_t *xs,
                   int score_only, const int32_t *subset, int64_t nsub, int known_multi_maxn,
                   int lane) {
    g_last_launches = 0;
    if (subset && nsub == 0) return TPZ_OK;
    if (n < 0 || n > INT32_MAX / 3 || !mat) { set_error("tpz_sw_batch: bad n or matrix"); return TPZ_E_ARG; }
    if (!(go > ge && ge >= 0 && go <= 255)) {
        set_error("tpz_sw_batch: requires 255 >= gap_open > gap_extend >= 0");
        return TPZ_E_ARG;
    }
    if (n == 0) return TPZ_OK;
    if (!q || !qoff || !qlen || !s || !soff || !slen || !score || !ref_end || !read_end || !status) {
        set_error("tpz_sw_batch: NULL buffer");
        return TPZ_E_ARG;
    }
    const LaunchCfg *cfg = nullptr;
    int rc = launch_cfg(&cfg, lane);
    if (rc) return rc;
    keep_pool_memory();

    // workspace: counts, cursor, rinfo, next_task, rerun_count, multi_maxn,
    // exact_count, (n_sub), per-bin rerun counts, i16 task counters | sorted,
    // rerun, exact_list
    const size_t small = sizeof(int32_t) * (2 * kBins + 2 * kRBins + kRBins + 8 + 2 * kRBins);
    const size_t bytes = small + sizeof(int32_t) * 3 * (size_t)n;
    char *ws = nullptr;
    TPZ_CUDA(cudaMallocAsync((void **)&ws, bytes, st));
    int32_t *counts = (int32_t *)ws;
    int32_t *cursor = counts + kBins;
    int32_t *rinfo = cursor + kBins;
    int32_t *next_task = rinfo + 2 * kRBins;
    int32_t *rerun_count = next_task + kRBins;
    int32_t *multi_maxn = rerun_count + 1;
    int32_t *exact_count = rerun_count + 2;
    int32_t *rerun_bin_count = rerun_count + 8;
    int32_t *next_task16 = rerun_bin_count + kRBins;
    int32_t *sorted = (int32_t *)(ws + small);
    int32_t *rerun = sorted + n;
    int32_t *exact_list = rerun + n;

    Args a;
    a.q = q; a.qoff = qoff; a.qlen = qlen; a.s = s; a.soff = soff; a.slen = slen;
    a.score = score; a.ref_end = ref_end; a.read_end = read_end; a.status = status;
    a.sorted = sorted; a.rinfo = rinfo; a.next_task = next_task;
    a.rerun = rerun; a.rerun_count = rerun_count;
    a.gap_open = go; a.gap_extend = ge;
    int mn = 0, mx = 0;
    for (int i = 0; i < 625; ++i) { mn = std::min<int>(mn, mat[i]); mx = std::max<int>(mx, mat[i]); }
    a.bias = -mn;
    memcpy(a.mat, mat, 625);
    a.translate = (xq && xs) ? 1 : 0;
    a.score_only = score_only;
    memset(a.xq, 0, sizeof a.xq);
    memset(a.xs, 0, sizeof a.xs);
    if (a.translate) {
        memcpy(a.xq, xq, 128);
        memcpy(a.xs, xs, 128);
    }
    a.bnd = nullptr;
    a.bnd_words = 0;
    a.exact_list = exact_list;
    a.exact_count = exact_count;
    a.exact_threshold = std::min(32767 - 2 * std::max(mx, 1), kBig);
    a.rerun_bin_count = rerun_bin_count;
    a.task_count = nullptr;
    // the i16 pass of a bin: its saturated pairs, in the bin's slice of rerun
    Args a16 = a;
    a16.ssw_lanes = 8;
    a16.sorted = rerun;
    a16.task_count = rerun_bin_count;
    a16.next_task = next_task16;
    a16.rerun_bin_count = nullptr;

    int64_t launches = 0;
    int host_maxn = 0;
    TPZ_CUDA(cudaMemsetAsync(rerun_count, 0, (8 + 2 * kRBins) * sizeof(int32_t), st));
    a.ssw_lanes = 16;
    if (subset) {
        // the first round over the given pair ids only
        int32_t *d_nsub = rerun_count + 3;
        set_i32_kernel<<<1, 1, 0, st>>>(d_nsub, (int32_t)nsub);
        rc = launch_round(cfg, a, nsub, subset, d_nsub, counts, cursor, sorted, multi_maxn, st,
                          launches, &host_maxn, -1, &a16);
    } else {
        rc = launch_round(cfg, a, n, nullptr, nullptr, counts, cursor, sorted, multi_maxn, st,
                          launches, &host_maxn, known_multi_maxn, &a16);
    }
    if (rc == TPZ_OK && (host_maxn > 0 || (int64_t)kStripeRows * mx >= a.exact_threshold)) {
        // only queries longer than one stripe, or matrices with large
        // entries, can come near the 16-bit limit
        int32_t *scratch = nullptr;
        rc = cudaMallocAsync((void **)&scratch,
                             sizeof(int32_t) * 2 * (size_t)TPZ_SW_MAX_QLEN * kExactThreads, st)
                 == cudaSuccess ? TPZ_OK : cuda_fail(cudaGetLastError(), "exact scratch");
        if (rc == TPZ_OK) {
            sw_exact_kernel<<<1, kExactThreads, 0, st>>>(a, scratch);
            ++launches;
            cudaFreeAsync(scratch, st);
        }
    }
    if (a.bnd) cudaFreeAsync(a.bnd, st);
    if (rc) { cudaFreeAsync(ws, st); return rc; }
    TPZ_CUDA(cudaFreeAsync(ws, st));
    TPZ_CUDA(cudaGetLastError());
    g_last_launches = launches;
    return TPZ_OK;
}

// Per host thread and device: launch attributes of the query-major kernels
// and two streams of their own, so that they run beside the pair-per-task
// kernels of the same call.
struct QmCfg {
    typedef void (*Fn)(const Args, QmArgs, int);
    Fn fn[2][kMaxR];                    // [score only][R - 1]
    int blocks_per_sm[2][kMaxR];
    cudaStream_t aux[kQmStreams];
    cudaEvent_t fork, join[kQmStreams];
};

template <int R>
struct QmTable {
    static void fill(QmCfg::Fn (*k)[kMaxR]) {
        k[0][R - 1] = sw_query_kernel<R, false>;
        k[1][R - 1] = sw_query_kernel<R, true>;
        QmTable<R - 1>::fill(k);
    }
};
template <>
struct QmTable<0> {
    static void fill(QmCfg::Fn (*)[kMaxR]) {}
};

struct QmCfgs {
    std::vector<QmCfg *> per_dev;
    ~QmCfgs() {
        for (QmCfg *c : per_dev) {
            if (!c) continue;
            for (int i = 0; i < kQmStreams; ++i) { cudaStreamDestroy(c->aux[i]); cudaEventDestroy(c->join[i]); }
            cudaEventDestroy(c->fork);
            delete c;
        }
    }
};

static int qm_cfg(const QmCfg **out) {
    static thread_local QmCfgs cfgs;
    int dev = 0;
    TPZ_CUDA(cudaGetDevice(&dev));
    if ((int)cfgs.per_dev.size() <= dev) cfgs.per_dev.resize(dev + 1, nullptr);
    if (!cfgs.per_dev[dev]) {
        QmCfg *c = new QmCfg();
        QmTable<kMaxR>::fill(c->fn);
        for (int so = 0; so < 2; ++so)
            for (int r = 1; r <= kMaxR; ++r) {
                const void *f = (const void *)c->fn[so][r - 1];
                TPZ_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              qm_smem_bytes(r)));
                TPZ_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                              (int)cudaSharedmemCarveoutMaxShared));
                int nb = 0;
                TPZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, kQmWarps * 32,
                                                                       qm_smem_bytes(r)));
                c->blocks_per_sm[so][r - 1] = std::max(1, nb);
            }
        for (int i = 0; i < kQmStreams; ++i) {
            TPZ_CUDA(cudaStreamCreateWithFlags(&c->aux[i], cudaStreamNonBlocking));
            TPZ_CUDA(cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming));
        }
        TPZ_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
        cfgs.per_dev[dev] = c;
    }
    *out = cfgs.per_dev[dev];
    return TPZ_OK;
}

int batch_device_grouped(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                         const int8_t *s, const int64_t *soff, const int32_t *slen,
                         const int8_t *mat, int go, int ge, int32_t *score, int32_t *ref_end,
                         int32_t *read_end, int32_t *status, cudaStream_t st, const int8_t *xq,
                         const int8_t *xs, int score_only, int64_t ngroups,
                         const int64_t *gstart_dev, const int64_t *gstart_host,
                         const int32_t *gqlen_host) {
    if (n <= 0) return TPZ_OK;
    if (!(go > ge && ge >= 0 && go <= 255) || !mat) {
        set_error("tpz_sw_batch: requires 255 >= gap_open > gap_extend >= 0");
        return TPZ_E_ARG;
    }
    // chunks of at most kQmMaxPairs pairs of one query for the query-major
    // kernels (queries with enough pairs and one stripe); every other pair
    // goes by pair
    std::vector<std::vector<int64_t>> per_r(kMaxR);
    std::vector<int64_t> work(kMaxR, 0);
    std::vector<int32_t> rest;
    for (int64_t g = 0; g < ngroups; ++g) {
        const int64_t c = gstart_host[g + 1] - gstart_host[g];
        if (c <= 0) continue;
        const int ql = gqlen_host[g];
        if (ql >= 1 && ql <= kStripeRows && c >= kQmMinPairs) {
            const int64_t nch = (c + kQmMaxPairs - 1) / kQmMaxPairs;
            for (int64_t i = 0; i < nch; ++i) {
                // equal cuts so that no chunk is much smaller than the others
                per_r[(ql + 31) / 32 - 1].push_back(gstart_host[g] + c * i / nch);
                per_r[(ql + 31) / 32 - 1].push_back(gstart_host[g] + c * (i + 1) / nch);
            }
            work[(ql + 31) / 32 - 1] += c * ql;
        } else {
            for (int64_t k = gstart_host[g]; k < gstart_host[g + 1]; ++k) rest.push_back((int32_t)k);
        }
    }
    std::vector<int64_t> chunks;
    std::vector<int32_t> bin_info(2 * kMaxR, 0);
    for (int r = 0; r < kMaxR; ++r) {
        bin_info[2 * r] = (int32_t)(chunks.size() / 2);
        bin_info[2 * r + 1] = (int32_t)(per_r[r].size() / 2);
        chunks.insert(chunks.end(), per_r[r].begin(), per_r[r].end());
    }
    const QmCfg *qc = nullptr;
    int rc = qm_cfg(&qc);
    if (rc) return rc;
    int64_t *dchunks = nullptr;
    int32_t *dbin = nullptr, *dnext = nullptr, *drest = nullptr, *dexact = nullptr,
            *dexact_n = nullptr;
    auto cleanup = [&]() {
        for (void *p : {(void *)dchunks, (void *)dbin, (void *)dnext, (void *)drest, (void *)dexact,
                        (void *)dexact_n})
            if (p) cudaFreeAsync(p, st);
    };
    if (cudaMallocAsync((void **)&dchunks, 8 * std::max<size_t>(chunks.size(), 1), st) ||
        cudaMallocAsync((void **)&dbin, 4 * 2 * kMaxR, st) ||
        cudaMallocAsync((void **)&dnext, 4 * kMaxR, st) ||
        cudaMallocAsync((void **)&drest, 4 * std::max<size_t>(rest.size(), 1), st) ||
        cudaMallocAsync((void **)&dexact, 4 * std::max<int64_t>(n, 1), st) ||
        cudaMallocAsync((void **)&dexact_n, 4, st)) {
        cleanup();
        return cuda_fail(cudaGetLastError(), "batch_device_grouped");
    }
    if (cudaMemcpyAsync(dchunks, chunks.data(), 8 * chunks.size(), cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(dbin, bin_info.data(), 4 * 2 * kMaxR, cudaMemcpyHostToDevice, st) ||
        cudaMemsetAsync(dnext, 0, 4 * kMaxR, st) || cudaMemsetAsync(dexact_n, 0, 4, st) ||
        (rest.size() && cudaMemcpyAsync(drest, rest.data(), 4 * rest.size(), cudaMemcpyHostToDevice, st))) {
        cleanup();
        return cuda_fail(cudaGetLastError(), "batch_device_grouped copies");
    }
    Args a;
    a.rerun_bin_count = nullptr;
    a.task_count = nullptr;
    memset(&a, 0, sizeof a);
    a.q = q; a.qoff = qoff; a.qlen = qlen; a.s = s; a.soff = soff; a.slen = slen;
    a.score = score; a.ref_end = ref_end; a.read_end = read_end; a.status = status;
    a.gap_open = go; a.gap_extend = ge;
    int mn = 0, mx = 0;
    for (int i = 0; i < 625; ++i) { mn = std::min<int>(mn, mat[i]); mx = std::max<int>(mx, mat[i]); }
    a.bias = -mn;
    memcpy(a.mat, mat, 625);
    a.translate = (xq && xs) ? 1 : 0;
    if (a.translate) { memcpy(a.xq, xq, 128); memcpy(a.xs, xs, 128); }
    a.score_only = score_only;
    a.exact_list = dexact;
    a.exact_count = dexact_n;
    a.exact_threshold = std::min(32767 - 2 * std::max(mx, 1), kBig);
    QmArgs g;
    g.chunks = dchunks; g.bin_info = dbin; g.next = dnext;
    const int nsm = sm_count();
    int64_t launches = 0;
    if (!chunks.empty()) {
        // one persistent kernel per row bin, the bins with the most work
        // first, over kQmStreams streams so that bins share the SMs
        TPZ_CUDA(cudaEventRecord(qc->fork, st));
        for (int i = 0; i < kQmStreams; ++i) TPZ_CUDA(cudaStreamWaitEvent(qc->aux[i], qc->fork, 0));
        std::vector<int> order;
        for (int r = 1; r <= kMaxR; ++r) if (!per_r[r - 1].empty()) order.push_back(r);
        std::sort(order.begin(), order.end(), [&](int x, int y) { return work[x - 1] > work[y - 1]; });
        int k = 0;
        const int so = a.score_only ? 1 : 0;
        for (int r : order) {
            const int grid = (int)std::min<int64_t>((int64_t)nsm * qc->blocks_per_sm[so][r - 1],
                                                    (int64_t)per_r[r - 1].size() / 2);
            qc->fn[so][r - 1]<<<grid, kQmWarps * 32, qm_smem_bytes(r), qc->aux[k++ % kQmStreams]>>>(
                a, g, r - 1);
            ++launches;
        }
    }
    rc = batch_device_x(n, q, qoff, qlen, s, soff, slen, mat, go, ge, score, ref_end, read_end,
                        status, st, xq, xs, score_only, drest, (int64_t)rest.size());
    launches += g_last_launches;
    if (!chunks.empty()) {
        for (int i = 0; i < kQmStreams; ++i) {
            TPZ_CUDA(cudaEventRecord(qc->join[i], qc->aux[i]));
            TPZ_CUDA(cudaStreamWaitEvent(st, qc->join[i], 0));
        }
        if (rc == TPZ_OK && (int64_t)kStripeRows * mx >= a.exact_threshold) {
            int32_t *scratch = nullptr;
            rc = cudaMallocAsync((void **)&scratch,
                                 sizeof(int32_t) * 2 * (size_t)TPZ_SW_MAX_QLEN * kExactThreads, st)
                     == cudaSuccess ? TPZ_OK : cuda_fail(cudaGetLastError(), "exact scratch");
            if (rc == TPZ_OK) {
                sw_exact_kernel<<<1, kExactThreads, 0, st>>>(a, scratch);
                ++launches;
                cudaFreeAsync(scratch, st);
            }
        }
    }
    cleanup();
    if (rc) return rc;
    TPZ_CUDA(cudaGetLastError());
    g_last_launches = launches;
    return TPZ_OK;
}

int batch_device(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                 const int8_t *s, const int64_t *soff, const int32_t *slen, const int8_t *mat,
                 int go, int ge, int32_t *score, int32_t *ref_end, int32_t *read_end,
                 int32_t *status, cudaStream_t st) {
    return batch_device_x(n, q, qoff, qlen, s, soff, slen, mat, go, ge, score, ref_end, read_end,
                          status, st, nullptr, nullptr, 0, nullptr, 0);
}

}  // namespace sw
}  // namespace tpz

// ------------------------------------------------------------------ C ABI

namespace {

// Grow-only device buffers reused by the host entry point, and its streams:
// two for the kernels (one per chunk), one for host-to-device and one for
// device-to-host copies, so that a chunk's copies run beside another
// chunk's kernels.
struct HostBatchBuffers {
    void *p = nullptr;
    size_t cap = 0;
    int dev = -1;
    cudaStream_t compute = nullptr, compute2 = nullptr, h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev[8] = {};
};
thread_local HostBatchBuffers g_hb;

int ensure(size_t bytes) {
    int dev = 0;
    TPZ_CUDA(cudaGetDevice(&dev));
    if (g_hb.compute && g_hb.dev != dev) {
        // streams and events belong to the device they were made on
        cudaStreamDestroy(g_hb.compute);
        cudaStreamDestroy(g_hb.compute2);
        cudaStreamDestroy(g_hb.h2d);
        cudaStreamDestroy(g_hb.d2h);
        for (cudaEvent_t &e : g_hb.ev) { cudaEventDestroy(e); e = nullptr; }
        g_hb.compute = g_hb.compute2 = g_hb.h2d = g_hb.d2h = nullptr;
    }
    if (!g_hb.compute) {
        TPZ_CUDA(cudaStreamCreateWithFlags(&g_hb.compute, cudaStreamNonBlocking));
        TPZ_CUDA(cudaStreamCreateWithFlags(&g_hb.compute2, cudaStreamNonBlocking));
        TPZ_CUDA(cudaStreamCreateWithFlags(&g_hb.h2d, cudaStreamNonBlocking));
        TPZ_CUDA(cudaStreamCreateWithFlags(&g_hb.d2h, cudaStreamNonBlocking));
        for (cudaEvent_t &e : g_hb.ev) TPZ_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (g_hb.p && (g_hb.cap >= bytes) && g_hb.dev == dev) return TPZ_OK;
    if (g_hb.p) cudaFree(g_hb.p);
    g_hb.p = nullptr;
    g_hb.cap = 0;
    TPZ_CUDA(cudaMalloc(&g_hb.p, bytes));
    g_hb.cap = bytes;
    g_hb.dev = dev;
    return TPZ_OK;
}

// Residue byte ranges [lo, hi) of q and s that the pairs [i0, i1) read, and
// the first pair outside the limits (-1: none).
struct Span {
    int64_t qlo, qhi, slo, shi, bad;
    int multi_maxn;     // longest subject of a pair whose query spans several stripes
};

Span scan_pairs(int64_t i0, int64_t i1, const int64_t *qoff, const int32_t *qlen,
                const int64_t *soff, const int32_t *slen) {
    Span r{INT64_MAX, 0, INT64_MAX, 0, -1, 0};
    for (int64_t i = i0; i < i1; ++i) {
        if (qlen[i] < 1 || qlen[i] > TPZ_SW_MAX_QLEN || slen[i] < 0 || slen[i] >= TPZ_SW_MAX_SLEN ||
            qoff[i] < 0 || soff[i] < 0) {
            r.bad = i;
            return r;
        }
        if (qlen[i] > tpz::sw::kStripeRows) r.multi_maxn = std::max(r.multi_maxn, slen[i]);
        r.qlo = std::min(r.qlo, qoff[i]);
        r.qhi = std::max(r.qhi, qoff[i] + qlen[i]);
        if (slen[i] > 0) {
            r.slo = std::min(r.slo, soff[i]);
            r.shi = std::max(r.shi, soff[i] + slen[i]);
        }
    }
    if (r.slo > r.shi) r.slo = r.shi;
    return r;
}

}  // namespace

namespace tpz {
namespace sw {

constexpr int kOneMaxQlen = kStripeRows;

typedef void (*OneFn)(const Args, int, int);

template <int R>
struct OneTable {
    static void fill(OneFn *k) {
        k[R - 1] = sw_one_kernel<R>;
        OneTable<R - 1>::fill(k);
    }
};
template <>
struct OneTable<0> {
    static void fill(OneFn *) {}
};

struct OneCfg {
    OneFn fn[kMaxR];
};

static int one_cfg(const OneCfg **out) {
    static std::mutex mu;
    static std::vector<OneCfg *> per_dev;
    int dev = 0;
    TPZ_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if ((int)per_dev.size() <= dev) per_dev.resize(dev + 1, nullptr);
    if (!per_dev[dev]) {
        OneCfg *c = new OneCfg();
        OneTable<kMaxR>::fill(c->fn);
        for (int r = 1; r <= kMaxR; ++r)
            TPZ_CUDA(cudaFuncSetAttribute((const void *)c->fn[r - 1],
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          smem_bytes(r)));
        per_dev[dev] = c;
    }
    *out = per_dev[dev];
    return TPZ_OK;
}

}  // namespace sw
}  // namespace tpz

extern "C" {

int tpz_sw_batch_device(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                        const int8_t *s, const int64_t *soff, const int32_t *slen,
                        const int8_t *mat625_host, int gap_open, int gap_extend,
                        int32_t *score, int32_t *ref_end, int32_t *read_end, int32_t *status,
                        void *stream) {
    return tpz::sw::batch_device(n, q, qoff, qlen, s, soff, slen, mat625_host, gap_open,
                                 gap_extend, score, ref_end, read_end, status,
                                 (cudaStream_t)stream);
}

int tpz_sw_batch_host(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                      const int8_t *s, const int64_t *soff, const int32_t *slen,
                      const int8_t *mat625, int gap_open, int gap_extend,
                      int32_t *score, int32_t *ref_end, int32_t *read_end, int32_t *status) {
    if (n < 0 || !mat625) { tpz::set_error("tpz_sw_batch_host: n < 0 or NULL matrix"); return TPZ_E_ARG; }
    if (!(gap_open > gap_extend && gap_extend >= 0 && gap_open <= 255)) {
        tpz::set_error("tpz_sw_batch_host: requires 255 >= gap_open > gap_extend >= 0");
        return TPZ_E_ARG;
    }
    if (n == 0) return TPZ_OK;
    // Pairs go in three chunks of 1/16, 3/16 and 12/16 of the batch: the copy
    // in of the inputs runs about six times faster than the kernels, so each
    // chunk's inputs arrive while the chunk before it computes and the GPU
    // waits only for the first sixteenth.  Consecutive chunks run on
    // alternating streams (lanes), so a chunk's kernels fill the GPU while
    // the previous chunk's last tasks finish; each chunk's results are
    // copied out as soon as they are done.  (Four chunks from 1/64 measured
    // 3 % slower: a small chunk still pays its longest task twice.)
    constexpr int kMaxChunks = 4;
    int64_t cut[kMaxChunks + 1] = {0, n};
    int nch = 1;
    if (n >= 65536) {
        cut[1] = n / 16; cut[2] = 4 * (n / 16); cut[3] = n;
        nch = 3;
    }
    // host-side validation and the byte ranges each chunk reads: the chunks
    // cut into pieces in proportion to their size, scanned on up to 16 host
    // threads, and merged per chunk
    Span sp[kMaxChunks];
    {
        const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        struct Piece { int c; int64_t i0, i1; Span r; };
        std::vector<Piece> pieces;
        for (int c = 0; c < nch; ++c) {
            const int64_t m = cut[c + 1] - cut[c];
            // at least 32,768 pairs per piece: a thread costs more than that
            const int64_t k = std::max<int64_t>(1, std::min((nt * m + n - 1) / n, m / 32768));
            for (int64_t p = 0; p < k; ++p)
                pieces.push_back({c, cut[c] + m * p / k, cut[c] + m * (p + 1) / k, Span{}});
        }
        std::vector<std::thread> th;
        for (size_t p = 1; p < pieces.size(); ++p)
            th.emplace_back([&, p]() {
                pieces[p].r = scan_pairs(pieces[p].i0, pieces[p].i1, qoff, qlen, soff, slen);
            });
        pieces[0].r = scan_pairs(pieces[0].i0, pieces[0].i1, qoff, qlen, soff, slen);
        for (auto &t : th) t.join();
        for (int c = 0; c < nch; ++c) sp[c] = Span{INT64_MAX, 0, INT64_MAX, 0, -1, 0};
        for (const Piece &p : pieces) {
            Span &d = sp[p.c];
            const Span &r = p.r;
            if (r.bad >= 0 && (d.bad < 0 || r.bad < d.bad)) d.bad = r.bad;
            d.multi_maxn = std::max(d.multi_maxn, r.multi_maxn);
            if (p.i1 > p.i0) {
                d.qlo = std::min(d.qlo, r.qlo);
                d.qhi = std::max(d.qhi, r.qhi);
                if (r.shi > r.slo || r.shi > 0) {
                    d.slo = std::min(d.slo, r.slo);
                    d.shi = std::max(d.shi, r.shi);
                }
            }
        }
        for (int c = 0; c < nch; ++c)
            if (sp[c].slo > sp[c].shi) sp[c].slo = sp[c].shi;
    }
    int64_t qbytes = 0, sbytes = 0;
    for (int c = 0; c < nch; ++c) {
        if (sp[c].bad >= 0) {
            const int64_t i = sp[c].bad;
            char buf[160];
            snprintf(buf, sizeof buf, "tpz_sw_batch_host: pair %lld outside the limits (qlen %d, slen %d)",
                     (long long)i, qlen[i], slen[i]);
            tpz::set_error(buf);
            return TPZ_E_RANGE;
        }
        qbytes = std::max(qbytes, sp[c].qhi);
        sbytes = std::max(sbytes, sp[c].shi);
    }
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t bq = al(qbytes), bs = al(sbytes), b8 = al(8 * (size_t)n), b4 = al(4 * (size_t)n);
    const size_t total = bq + bs + 2 * b8 + 6 * b4;
    int rc = ensure(total);
    if (rc) return rc;
    char *d = (char *)g_hb.p;
    int8_t *dq = (int8_t *)d; d += bq;
    int8_t *ds = (int8_t *)d; d += bs;
    int64_t *dqoff = (int64_t *)d; d += b8;
    int64_t *dsoff = (int64_t *)d; d += b8;
    int32_t *dqlen = (int32_t *)d; d += b4;
    int32_t *dslen = (int32_t *)d; d += b4;
    int32_t *dsc = (int32_t *)d; d += b4;
    int32_t *dre = (int32_t *)d; d += b4;
    int32_t *drd = (int32_t *)d; d += b4;
    int32_t *dst = (int32_t *)d; d += b4;
    cudaStream_t cst[2] = {g_hb.compute, g_hb.compute2}, hs = g_hb.h2d, os = g_hb.d2h;
    // The device copies of q and s keep the host offsets.  Each chunk copies
    // the part of its byte range not copied yet: the copied part is kept as
    // one interval [lo, hi) that grows to cover every range seen (a gap
    // between ranges is copied too, which is harmless).
    int64_t qc_lo = 0, qc_hi = 0, sc_lo = 0, sc_hi = 0;
    auto copy_new = [&](const int8_t *src, int8_t *dst, int64_t lo, int64_t hi, int64_t &c_lo,
                        int64_t &c_hi) -> cudaError_t {
        if (hi <= lo) return cudaSuccess;
        if (c_hi <= c_lo) {
            c_lo = lo; c_hi = hi;
            return cudaMemcpyAsync(dst + lo, src + lo, hi - lo, cudaMemcpyHostToDevice, hs);
        }
        cudaError_t e = cudaSuccess;
        if (lo < c_lo) {
            e = cudaMemcpyAsync(dst + lo, src + lo, c_lo - lo, cudaMemcpyHostToDevice, hs);
            c_lo = lo;
        }
        if (e == cudaSuccess && hi > c_hi) {
            e = cudaMemcpyAsync(dst + c_hi, src + c_hi, hi - c_hi, cudaMemcpyHostToDevice, hs);
            c_hi = hi;
        }
        return e;
    };
    static_assert(2 * kMaxChunks <= (int)(sizeof g_hb.ev / sizeof g_hb.ev[0]), "events per chunk");
    cudaEvent_t *in_ready = g_hb.ev, *done = g_hb.ev + kMaxChunks;
    for (int c = 0; c < nch; ++c) {
        const int64_t a = cut[c], m = cut[c + 1] - cut[c];
        TPZ_CUDA(copy_new(q, dq, sp[c].qlo, sp[c].qhi, qc_lo, qc_hi));
        TPZ_CUDA(copy_new(s, ds, sp[c].slo, sp[c].shi, sc_lo, sc_hi));
        TPZ_CUDA(cudaMemcpyAsync(dqoff + a, qoff + a, 8 * m, cudaMemcpyHostToDevice, hs));
        TPZ_CUDA(cudaMemcpyAsync(dsoff + a, soff + a, 8 * m, cudaMemcpyHostToDevice, hs));
        TPZ_CUDA(cudaMemcpyAsync(dqlen + a, qlen + a, 4 * m, cudaMemcpyHostToDevice, hs));
        TPZ_CUDA(cudaMemcpyAsync(dslen + a, slen + a, 4 * m, cudaMemcpyHostToDevice, hs));
        TPZ_CUDA(cudaEventRecord(in_ready[c], hs));
    }
    for (int c = 0; c < nch; ++c) {
        const int64_t a = cut[c], m = cut[c + 1] - cut[c];
        cudaStream_t cs = cst[c & 1];
        TPZ_CUDA(cudaStreamWaitEvent(cs, in_ready[c], 0));
        rc = tpz::sw::batch_device_x(m, dq, dqoff + a, dqlen + a, ds, dsoff + a, dslen + a,
                                     mat625, gap_open, gap_extend, dsc + a, dre + a, drd + a,
                                     dst + a, cs, nullptr, nullptr, 0, nullptr, 0,
                                     sp[c].multi_maxn, c & 1);
        if (rc) {
            cudaStreamSynchronize(hs);
            cudaStreamSynchronize(cst[0]);
            cudaStreamSynchronize(cst[1]);
            return rc;
        }
        TPZ_CUDA(cudaEventRecord(done[c], cs));
        TPZ_CUDA(cudaStreamWaitEvent(os, done[c], 0));
        TPZ_CUDA(cudaMemcpyAsync(score + a, dsc + a, 4 * m, cudaMemcpyDeviceToHost, os));
        TPZ_CUDA(cudaMemcpyAsync(ref_end + a, dre + a, 4 * m, cudaMemcpyDeviceToHost, os));
        TPZ_CUDA(cudaMemcpyAsync(read_end + a, drd + a, 4 * m, cudaMemcpyDeviceToHost, os));
        TPZ_CUDA(cudaMemcpyAsync(status + a, dst + a, 4 * m, cudaMemcpyDeviceToHost, os));
    }
    TPZ_CUDA(cudaStreamSynchronize(os));
    TPZ_CUDA(cudaStreamSynchronize(cst[0]));
    TPZ_CUDA(cudaStreamSynchronize(cst[1]));
    return TPZ_OK;
}

int64_t tpz_sw_last_launches(void) { return tpz::sw::g_last_launches; }

int tpz_sw_align_one(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                     const int8_t *mat625_host, int gap_open, int gap_extend, int32_t *out4,
                     void *stream) {
    using namespace tpz::sw;
    if (!q || !s || !out4 || !mat625_host || qlen < 1 || qlen > kOneMaxQlen || slen < 0 ||
        slen >= TPZ_SW_MAX_SLEN) {
        tpz::set_error("tpz_sw_align_one: need 1 <= qlen <= 1024, 0 <= slen < 2^24, non-NULL buffers");
        return TPZ_E_ARG;
    }
    if (!(gap_open > gap_extend && gap_extend >= 0 && gap_open <= 255)) {
        tpz::set_error("tpz_sw_align_one: requires 255 >= gap_open > gap_extend >= 0");
        return TPZ_E_ARG;
    }
    const OneCfg *cfg = nullptr;
    int rc = one_cfg(&cfg);
    if (rc) return rc;
    int mn = 0, mx = 0;
    for (int i = 0; i < 625; ++i) { mn = std::min<int>(mn, mat625_host[i]); mx = std::max<int>(mx, mat625_host[i]); }
    if ((int64_t)qlen * mx >= kBig) {
        tpz::set_error("tpz_sw_align_one: matrix entries too large for 16-bit scores at this length");
        return TPZ_E_ARG;
    }
    Args a;
    a.rerun_bin_count = nullptr;
    a.task_count = nullptr;
    memset(&a, 0, sizeof a);
    a.q = q; a.s = s;
    a.score = out4; a.ref_end = out4 + 1; a.read_end = out4 + 2; a.status = out4 + 3;
    a.gap_open = gap_open; a.gap_extend = gap_extend; a.bias = -mn;
    memcpy(a.mat, mat625_host, 625);
    a.exact_threshold = 32767;
    const int R = (qlen + 31) / 32;
    cfg->fn[R - 1]<<<1, 32, smem_bytes(R), (cudaStream_t)stream>>>(a, qlen, slen);
    TPZ_CUDA(cudaGetLastError());
    return TPZ_OK;
}

int tpz_dpx_probe(int64_t blocks, int iters, uint32_t *out, void *stream, int64_t *ops) {
    if (blocks < 1 || iters < 1 || !out || !ops) { tpz::set_error("tpz_dpx_probe: bad argument"); return TPZ_E_ARG; }
    tpz::sw::dpx_probe_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(
        iters, 0x00010001u, 0x80008000u, out);
    TPZ_CUDA(cudaGetLastError());
    *ops = blocks * 256 * (int64_t)iters * tpz::sw::kProbeChains;
    return TPZ_OK;
}

}  // extern "C"

// ------------------------------------------------- allocation-free variant
//
// Some callers cannot let a library allocate device memory on their request
// path: a search server that has planned its HBM around a resident index and
// a fixed set of in-flight batches (an allocation there can fail under
// memory pressure halfway through a request), or a host loop that must not
// stall on the allocator -- cudaMalloc/cudaFree synchronize the device and
// would serialize every concurrent stream.  For them the batched SW below
// keeps its scratch (bin counts, bin cursors, the sorted pair list and the
// rerun list) in one statically sized device array instead of a per-call
// allocation, and enqueues everything on the caller's stream only.

namespace tpz {
namespace sw {

constexpr int64_t kNoAllocMaxPairs = TPZ_SW_NOALLOC_MAX_PAIRS;
constexpr int kNoAllocMaxQlen = TPZ_SW_NOALLOC_MAX_QLEN;   // one stripe
// the stated entry limit is the largest one the 16-bit lanes hold exactly
static_assert((int64_t)kNoAllocMaxQlen * TPZ_SW_NOALLOC_MAX_ENTRY < kBig &&
                  (int64_t)kNoAllocMaxQlen * (TPZ_SW_NOALLOC_MAX_ENTRY + 1) >= kBig,
              "TPZ_SW_NOALLOC_MAX_ENTRY");
constexpr size_t kNoAllocWords = 2 * (size_t)kBins + 2 * kRBins + kRBins + 4 + 2 * (size_t)kNoAllocMaxPairs;

// One copy per device that loads the library, kept until the process exits.
static __device__ __align__(256) int32_t g_noalloc_scratch[kNoAllocWords];

struct NoAllocDev {
    int32_t *scratch = nullptr;      // device address of g_noalloc_scratch
    KernelFn fn[kMaxR];
    int blocks_per_sm[kMaxR];
};

// Per-device set-up, done by the first call on each device with that device
// current: the device address of the static scratch array (host code cannot
// use the array's name as a device pointer) and the bin kernels' launch
// attributes.
static int noalloc_setup(const NoAllocDev **out) {
    static std::mutex mu;
    static std::vector<NoAllocDev *> per_dev;
    int dev = 0;
    TPZ_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if ((int)per_dev.size() <= dev) per_dev.resize(dev + 1, nullptr);
    if (!per_dev[dev]) {
        NoAllocDev *d = new NoAllocDev();
        cudaError_t e = cudaGetSymbolAddress((void **)&d->scratch, g_noalloc_scratch);
        if (e != cudaSuccess) {
            delete d;
            return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        }
        Table<kMaxR>::fill(d->fn);
        for (int r = 1; r <= kMaxR; ++r) {
            e = cudaFuncSetAttribute((const void *)d->fn[r - 1],
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes(r));
            int nb = 0;
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void *)d->fn[r - 1], 32,
                                                                  smem_bytes(r));
            if (e != cudaSuccess) {
                delete d;
                return cuda_fail(e, "allocation-free SW set-up");
            }
            d->blocks_per_sm[r - 1] = std::max(1, nb);
        }
        per_dev[dev] = d;
    }
    *out = per_dev[dev];
    return TPZ_OK;
}

static int noalloc_round(const NoAllocDev *d, Args &a, int64_t n, const int32_t *list,
                         const int32_t *list_n, int32_t *counts, int32_t *cursor, int32_t *sorted,
                         cudaStream_t st) {
    const int nsm = sm_count();
    TPZ_CUDA(cudaMemsetAsync(counts, 0, sizeof(int32_t) * kBins, st));
    const int gb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)nsm * 8);
    bin_count_kernel<<<std::max(gb, 1), 256, 0, st>>>(n, list, list_n, a.qlen, a.slen, counts,
                                                      a.status, kNoAllocMaxQlen, nullptr);
    bin_scan_kernel<<<1, 1024, 0, st>>>(counts, cursor, const_cast<int32_t *>(a.rinfo), a.next_task);
    bin_scatter_kernel<<<std::max(gb, 1), 256, 0, st>>>(n, list, list_n, a.qlen, a.slen, cursor,
                                                        sorted, kNoAllocMaxQlen);
    for (int r = kMaxR; r >= 1; --r)
        d->fn[r - 1]<<<nsm * d->blocks_per_sm[r - 1], 32, smem_bytes(r), st>>>(a, r - 1, 1);
    TPZ_CUDA(cudaGetLastError());
    return TPZ_OK;
}

}  // namespace sw
}  // namespace tpz

extern "C" int tpz_sw_batch_device_noalloc(int64_t n, const int8_t *q, const int64_t *qoff,
                                           const int32_t *qlen, const int8_t *s,
                                           const int64_t *soff, const int32_t *slen,
                                           const int8_t *mat625_host, int gap_open,
                                           int gap_extend, int32_t *score, int32_t *ref_end,
                                           int32_t *read_end, int32_t *status, void *stream) {
    using namespace tpz::sw;
    if (n < 0 || !mat625_host) {
        tpz::set_error("tpz_sw_batch_device_noalloc: n < 0 or NULL matrix");
        return TPZ_E_ARG;
    }
    if (n > kNoAllocMaxPairs) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "tpz_sw_batch_device_noalloc: %lld pairs exceed the fixed scratch of %lld pairs; "
                 "split the batch or use tpz_sw_batch_device",
                 (long long)n, (long long)kNoAllocMaxPairs);
        tpz::set_error(buf);
        return TPZ_E_RANGE;
    }
    if (!(gap_open > gap_extend && gap_extend >= 0 && gap_open <= 255)) {
        tpz::set_error("tpz_sw_batch_device_noalloc: requires 255 >= gap_open > gap_extend >= 0");
        return TPZ_E_ARG;
    }
    if (n == 0) return TPZ_OK;
    if (!q || !qoff || !qlen || !s || !soff || !slen || !score || !ref_end || !read_end || !status) {
        tpz::set_error("tpz_sw_batch_device_noalloc: NULL buffer");
        return TPZ_E_ARG;
    }
    // 16-bit lanes are exact only while every score stays below the Fm
    // reset addend and clear of the int16 limit; a query of up to
    // kNoAllocMaxQlen rows can score at most kNoAllocMaxQlen * (largest
    // entry).  The allocating call re-runs such pairs in 32 bits with
    // scratch of its own; this one has none, so it refuses the matrix.
    int mn = 0, mx = 0;
    for (int i = 0; i < 625; ++i) {
        mn = std::min<int>(mn, mat625_host[i]);
        mx = std::max<int>(mx, mat625_host[i]);
    }
    if ((int64_t)kNoAllocMaxQlen * mx >= std::min(32767 - 2 * std::max(mx, 1), kBig)) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "tpz_sw_batch_device_noalloc: largest matrix entry %d is too large for exact "
                 "16-bit scores of %d-residue queries (limit %d); use tpz_sw_batch_device",
                 mx, kNoAllocMaxQlen, TPZ_SW_NOALLOC_MAX_ENTRY);
        tpz::set_error(buf);
        return TPZ_E_ARG;
    }
    const NoAllocDev *d = nullptr;
    int rc = noalloc_setup(&d);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int32_t *counts = d->scratch;
    int32_t *cursor = counts + kBins;
    int32_t *rinfo = cursor + kBins;
    int32_t *next_task = rinfo + 2 * kRBins;
    int32_t *rerun_count = next_task + kRBins;
    int32_t *sorted = rerun_count + 4;
    int32_t *rerun = sorted + kNoAllocMaxPairs;

    Args a;
    a.rerun_bin_count = nullptr;
    a.task_count = nullptr;
    a.q = q; a.qoff = qoff; a.qlen = qlen; a.s = s; a.soff = soff; a.slen = slen;
    a.score = score; a.ref_end = ref_end; a.read_end = read_end; a.status = status;
    a.sorted = sorted; a.rinfo = rinfo; a.next_task = next_task;
    a.rerun = rerun; a.rerun_count = rerun_count;
    a.gap_open = gap_open; a.gap_extend = gap_extend;
    a.bias = -mn;
    memcpy(a.mat, mat625_host, 625);
    a.translate = 0;
    a.score_only = 0;
    memset(a.xq, 0, sizeof a.xq);
    memset(a.xs, 0, sizeof a.xs);
    a.bnd = nullptr;
    a.bnd_words = 0;
    a.exact_list = nullptr;
    a.exact_count = nullptr;
    a.exact_threshold = 32767;

    // the rerun counter carries the previous call's value: clear it
    TPZ_CUDA(cudaMemsetAsync(rerun_count, 0, sizeof(int32_t), st));
    a.ssw_lanes = 16;
    rc = noalloc_round(d, a, n, nullptr, nullptr, counts, cursor, sorted, st);
    if (rc) return rc;
    a.ssw_lanes = 8;
    return noalloc_round(d, a, n, rerun, rerun_count, counts, cursor, sorted, st);
}
