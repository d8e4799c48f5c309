// stats_kernel.cu -- the --blasttab columns of reported hits on the device:
// start coordinates, alignment length, mismatches, gap opens and identity,
// with the results of ssw_align_stats (src/ssw.c:900-978, called per printed
// hit by stats_using_ssw_profile, src/ssw_wrapper.c:132-155, from
// query_perform_statistics, src/query.c:250-299).
//
// One thread per hit, two launches:
//
// 1. Start coordinates.  A local-alignment pass from the end cell backwards:
//    subject columns ref_end .. 0 against the query prefix read[0 .. read_end]
//    reversed, with the recurrence of SSW's striped passes (the in-lane F
//    term reset every `seg` rows, seg = ceil(rows / 16) when bias + score <
//    255 and ceil(rows / 8) otherwise, and padding rows past the query that
//    score 0 but still count toward a column's maximum), stopping at the
//    first column whose maximum equals the forward score.  The column and
//    row of the best cell give the subject and query starts.
//    Then the band search: a banded global-style pass over the aligned
//    segments (H never below 0 through its gap terms, cells outside the
//    band read as 0), the band starting at |len difference| + 1 and doubling
//    until the best cell reaches the score; it yields the final band and the
//    size of its direction table, or the size guard of the reference (a
//    table of 2^30 bytes or more gives -1 columns).
// 2. Path.  The band passes again, now writing per cell the step each of the
//    three states (vertical gap, horizontal gap, match) came from into a
//    table laid out row by row (2 * band + 1 cells of 3 bytes per row, the
//    passes of every band width writing the same table, as the reference's
//    reused buffer does), then the walk back from the end cell: counts of
//    columns, mismatches (residues compared after each diagonal step) and
//    gap opens, until the walk reaches the first query row or leaves its
//    row's slot.
#include <algorithm>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "search_internal.cuh"
#include "tpz_common.cuh"

namespace tpz {
namespace stats {

struct PairArgs {
    int64_t n;
    const int8_t *q, *s;                 // residues (matrix indices, or bytes through xmap)
    const int64_t *qoff, *soff;
    const int32_t *qlen, *slen;
    const int32_t *read_end, *ref_end, *score;   // forward pass results
    const int32_t *valid;                // nullptr, or nonzero for the pairs to do
    int8_t mat[625];
    int8_t xmap[128];
    int translate;
    int gap_open, gap_extend, bias;
    // outputs
    int32_t *qstart, *sstart, *length, *gapopen, *mismatch;
    double *identity;
    // per pair work state between the launches
    int32_t *band;                       // final band width, 0 = no banded pass
    int64_t *dir_bytes;                  // direction table size of the final band
    // scratch
    int32_t *work;                       // int32 arrays, per pair at work_off
    const int64_t *work_off;
    int8_t *dir;                         // direction tables, per pair at dir_off
    const int64_t *dir_off;
};

__device__ __forceinline__ int res_at(const PairArgs &a, const int8_t *p, int64_t i) {
    int v = p[i];
    if (a.translate) v = a.xmap[v & 127];
    return v;
}

// scratch words of a pair: reverse pass 3 * (rows + 1), band rows 2 * (cols + 2)
__host__ __device__ inline int64_t work_words(int32_t read_end, int32_t ref_end) {
    const int64_t n = (int64_t)read_end + 1;
    const int64_t rows = ((n + 15) / 16) * 16;
    return 3 * (rows + 1) + 2 * ((int64_t)ref_end + 3);
}

// the band rows' part of a pair's scratch starts after the reverse pass's
__host__ __device__ inline int64_t band_words_at(int32_t read_end) {
    const int64_t n = (int64_t)read_end + 1;
    return 3 * (((n + 15) / 16) * 16 + 1);
}

// One banded pass over query rows [0, rl) and subject columns [0, fl):
// H and E of the previous row live in Hc/Ec by column (cells outside the
// previous row's band read as 0); dir (may be null) receives the steps.
// Returns the pass's best cell.
__device__ int band_pass(const PairArgs &a, const int8_t *rd, const int8_t *rf, int rl, int fl,
                         int w, int32_t *Hc, int32_t *Ec, int8_t *dir) {
    const int go = a.gap_open, ge = a.gap_extend;
    const int64_t wd3 = (int64_t)(2 * w + 1) * 3;
    int best = 0;
    for (int j = 0; j < fl + 2; ++j) { Hc[j] = 0; Ec[j] = 0; }
    int prev_end = -1;
    for (int i = 0; i < rl; ++i) {
        const int beg = max(0, i - w), end = min(fl - 1, i + w);
        // the column past the previous row's band reads as 0
        if (prev_end + 1 < fl) { Hc[prev_end + 1] = 0; Ec[prev_end + 1] = 0; }
        const int qi = res_at(a, rd, i);
        int diag = beg > 0 ? Hc[beg - 1] : 0;      // H(i-1, beg-1), 0 outside
        int hl = 0, f = 0;                          // H(i, j-1), F(i, j-1)
        int8_t *dl = dir ? dir + (int64_t)i * wd3 : nullptr;
        for (int j = beg; j <= end; ++j) {
            const int hu = Hc[j], eu = Ec[j];           // previous row, column j
            const int eo = hu - go, ee = eu - ge;
            const int e = eo > ee ? eo : ee;
            const int fo = hl - go, fe = f - ge;
            f = fo > fe ? fo : fe;
            const int e1 = e > 0 ? e : 0, f1 = f > 0 ? f : 0;
            const int gap = e1 > f1 ? e1 : f1;
            const int dg = diag + a.mat[res_at(a, rf, j) * 25 + qi];
            const int h = gap > dg ? gap : dg;
            if (dl) {
                const int8_t de = eo > ee ? 3 : 2, df = fo > fe ? 5 : 4;
                int8_t *c = dl + (int64_t)(j - beg) * 3;
                c[0] = de;
                c[1] = df;
                c[2] = gap <= dg ? 1 : (e1 > f1 ? de : df);
            }
            best = h > best ? h : best;
            diag = hu;
            Hc[j] = h;
            Ec[j] = e;
            hl = h;
        }
        prev_end = end;
    }
    return best;
}

__global__ void stats_start_kernel(const __grid_constant__ PairArgs a) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n;
         p += (int64_t)gridDim.x * blockDim.x) {
        a.band[p] = 0;
        a.dir_bytes[p] = 0;
        if (a.valid && !a.valid[p]) continue;
        const int re = a.read_end[p], fe = a.ref_end[p], score = a.score[p];
        if (re < 0 || fe < 0) {
            a.qstart[p] = a.sstart[p] = a.length[p] = a.gapopen[p] = a.mismatch[p] = -1;
            a.identity[p] = -1.0;
            continue;
        }
        const int8_t *q = a.q + a.qoff[p], *s = a.s + a.soff[p];
        // ---- reverse pass: rows = reversed query prefix, columns fe .. 0
        const int n = re + 1;
        const bool word = !(a.bias + score < 255);
        const int lanes = word ? 8 : 16;
        const int seg = (n + lanes - 1) / lanes;
        const int rows = seg * lanes;
        const int terminate = word ? (score & 0xFFFF) : (score & 0xFF);
        int32_t *w = a.work + a.work_off[p];
        int32_t *E = w, *Hp = w + (rows + 1), *Hn = w + 2 * (rows + 1);
        for (int r = 0; r <= rows; ++r) { E[r] = 0; Hp[r] = 0; Hn[r] = 0; }
        const int go = a.gap_open, gx = a.gap_extend;
        int best = 0, bc = word ? 0 : -1, br = 0;
        for (int c = fe; c >= 0; --c) {
            const int8_t *mrow = a.mat + 25 * res_at(a, s, c);
            int F = 0, Fm = 0, colmax = 0, cbest = 0, crow = 0;
            for (int r = 0; r < rows; ++r) {
                if (r % seg == 0) Fm = 0;
                const int D = r ? Hp[r - 1] : 0;
                const int sc = r < n ? mrow[res_at(a, q, re - r)] : 0;
                const int hp = max(max(0, D + sc), max(E[r], Fm));
                const int h = max(hp, F);
                E[r] = max(0, max(E[r] - gx, hp - go));
                Fm = max(0, max(Fm - gx, hp - go));
                F = max(0, max(F - gx, h - go));
                Hn[r] = h;
                colmax = max(colmax, h);
                if (r < n && h > cbest) { cbest = h; crow = r; }
            }
            int32_t *t = Hp; Hp = Hn; Hn = t;
            if (cbest > best) {
                best = cbest;
                if ((!word && best + a.bias >= 255) || (word && best >= 32767)) break;
                bc = c;
                br = crow;
            }
            if (colmax == terminate) break;
        }
        const int rread = best > 0 ? br : 0;
        const int qs = re - rread, ss = bc;
        a.qstart[p] = qs;
        a.sstart[p] = ss;
        if (ss < 0) {
            a.length[p] = a.gapopen[p] = a.mismatch[p] = -1;
            a.identity[p] = -1.0;
            continue;
        }
        // ---- band search
        const int fl = fe - ss + 1, rl = re - qs + 1;
        int band = abs(fl - rl) + 1;
        int32_t *Hc = w + band_words_at(re), *Ec = Hc + (fe + 3);
        int mx = 0;
        bool guard = false;
        for (;;) {
            // the reference sizes its table as the power of two above this
            // and gives up (-1 columns) at 2^31
            const int64_t need = (int64_t)(2 * band + 1) * rl * 3;
            if (need >= ((int64_t)1 << 30)) { guard = true; break; }
            mx = max(mx, band_pass(a, q + qs, s + ss, rl, fl, band, Hc, Ec, nullptr));
            if (mx >= score) break;
            band *= 2;
        }
        if (guard) {
            a.length[p] = a.gapopen[p] = a.mismatch[p] = -1;
            a.identity[p] = -1.0;
            continue;
        }
        a.band[p] = band;
        a.dir_bytes[p] = (int64_t)(2 * band + 1) * rl * 3;
    }
}

__global__ void stats_path_kernel(const __grid_constant__ PairArgs a) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int wfinal = a.band[p];
        if (wfinal <= 0) continue;
        const int re = a.read_end[p], fe = a.ref_end[p];
        const int qs = a.qstart[p], ss = a.sstart[p];
        const int fl = fe - ss + 1, rl = re - qs + 1;
        const int8_t *rd = a.q + a.qoff[p] + qs, *rf = a.s + a.soff[p] + ss;
        int32_t *Hc = a.work + a.work_off[p] + band_words_at(re), *Ec = Hc + (fe + 3);
        int8_t *dir = a.dir + a.dir_off[p];
        // every band width up to the final one writes the same table
        for (int band = abs(fl - rl) + 1;; band *= 2) {
            band_pass(a, rd, rf, rl, fl, band, Hc, Ec, dir);
            if (band >= wfinal) break;
        }
        const int64_t wd3 = (int64_t)(2 * wfinal + 1) * 3;
        int i = rl - 1, j = fl - 1, st = 2, len = 0, mism = 0, gaps = 0, same = 0;
        char prev = 'M';
        bool broken = false;
        while (i > 0) {
            const int x = max(0, i - wfinal);
            const int64_t at = (int64_t)(j - x) * 3 + st;
            if (at < 0 || at >= wd3) break;              // left the row's slot
            char op;
            switch (dir[(int64_t)i * wd3 + at]) {
            case 1: --i; --j; st = 2; op = 'M'; break;
            case 2: --i; st = 0; op = 'I'; break;
            case 3: --i; st = 2; op = 'I'; break;
            case 4: --j; st = 1; op = 'D'; break;
            case 5: --j; st = 2; op = 'D'; break;
            default: broken = true; op = 0; break;
            }
            if (broken) break;
            if (op == 'M') {
                if (res_at(a, rd, i) != res_at(a, rf, j)) ++mism; else ++same;
            }
            if ((op == 'I' && prev != 'I') || (op == 'D' && prev != 'D')) ++gaps;
            ++len;
            prev = op;
        }
        a.length[p] = len;
        a.gapopen[p] = gaps;
        a.mismatch[p] = mism;
        a.identity[p] = broken ? 0.0 : same / (double)len;
    }
}

__global__ void work_words_kernel(int64_t n, const int32_t *read_end, const int32_t *ref_end,
                                  const int32_t *valid, int64_t *words) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const bool on = (!valid || valid[p]) && read_end[p] >= 0 && ref_end[p] >= 0;
        words[p] = on ? work_words(read_end[p], ref_end[p]) : 0;
    }
}

// exclusive offsets from sizes, with the total at [n]
int exclusive_offsets(const int64_t *size, int64_t n, int64_t *off, cudaStream_t st,
                      std::vector<void *> &mem, int64_t *total) {
    size_t tb = 0;
    TPZ_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, size, off, n, st));
    void *tmp = nullptr;
    TPZ_CUDA(cudaMallocAsync(&tmp, std::max<size_t>(tb, 16), st));
    mem.push_back(tmp);
    TPZ_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, size, off, n, st));
    int64_t last[2] = {0, 0};
    TPZ_CUDA(cudaMemcpyAsync(&last[0], off + n - 1, 8, cudaMemcpyDeviceToHost, st));
    TPZ_CUDA(cudaMemcpyAsync(&last[1], size + n - 1, 8, cudaMemcpyDeviceToHost, st));
    TPZ_CUDA(cudaStreamSynchronize(st));
    *total = last[0] + last[1];
    return TPZ_OK;
}

int stats_batch(PairArgs a, cudaStream_t st) {
    if (a.n <= 0) return TPZ_OK;
    std::vector<void *> mem;
    auto cleanup = [&]() { for (void *p : mem) cudaFreeAsync(p, st); };
    auto alloc = [&](void **p, size_t bytes) -> int {
        TPZ_CUDA(cudaMallocAsync(p, std::max<size_t>(bytes, 16), st));
        mem.push_back(*p);
        return TPZ_OK;
    };
    int rc;
    int64_t *words, *woff, *dbytes, *doff;
    int32_t *band;
    if ((rc = alloc((void **)&words, 8 * a.n)) || (rc = alloc((void **)&woff, 8 * a.n)) ||
        (rc = alloc((void **)&dbytes, 8 * a.n)) || (rc = alloc((void **)&doff, 8 * a.n)) ||
        (rc = alloc((void **)&band, 4 * a.n))) {
        cleanup();
        return rc;
    }
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((a.n + 127) / 128, 4096));
    work_words_kernel<<<grid, 128, 0, st>>>(a.n, a.read_end, a.ref_end, a.valid, words);
    int64_t total_words = 0;
    if ((rc = exclusive_offsets(words, a.n, woff, st, mem, &total_words))) { cleanup(); return rc; }
    int32_t *work;
    if ((rc = alloc((void **)&work, 4 * (size_t)total_words))) { cleanup(); return rc; }
    a.band = band; a.dir_bytes = dbytes; a.work = work; a.work_off = woff;
    // few hits per batch: small blocks spread them over the SMs
    stats_start_kernel<<<grid, 128, 0, st>>>(a);
    TPZ_CUDA(cudaGetLastError());
    int64_t total_dir = 0;
    if ((rc = exclusive_offsets(dbytes, a.n, doff, st, mem, &total_dir))) { cleanup(); return rc; }
    int8_t *dir;
    if ((rc = alloc((void **)&dir, (size_t)total_dir))) { cleanup(); return rc; }
    // never-written table cells read as "no step" (the walk stops there)
    TPZ_CUDA(cudaMemsetAsync(dir, 0, (size_t)total_dir, st));
    a.dir = dir; a.dir_off = doff;
    stats_path_kernel<<<grid, 128, 0, st>>>(a);
    TPZ_CUDA(cudaGetLastError());
    cleanup();
    return TPZ_OK;
}

// pair list of reported search hits: query text offset by query, subject
// offset by protein, forward results as reported, only SW-aligned hits
__global__ void reported_pairs_kernel(int64_t n, const int32_t *query_of, const int64_t *qoff_q,
                                      const int64_t *pstart, const int32_t *protein,
                                      const int32_t *sw_status, int64_t *qoff, int64_t *soff,
                                      int32_t *valid, int32_t *qstart, int32_t *sstart,
                                      int32_t *length, int32_t *gapopen, int32_t *mismatch,
                                      double *identity) {
    for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < n;
         d += (int64_t)gridDim.x * blockDim.x) {
        qoff[d] = qoff_q[query_of[d]];
        soff[d] = pstart[protein[d]];
        valid[d] = sw_status[d] == TPZ_SW_OK;
        qstart[d] = sstart[d] = length[d] = gapopen[d] = mismatch[d] = -1;
        identity[d] = -1.0;
    }
}

int reported_stats(int64_t n, const int8_t *qtext, const int64_t *qoff_q, const int32_t *query_of,
                   const int8_t *T, const int64_t *pstart, const int32_t *protein,
                   const int32_t *raw, const int32_t *qend, const int32_t *send,
                   const int32_t *sw_status, const int8_t *mat, const int8_t *xmap, int go, int ge,
                   int32_t *qstart, int32_t *sstart, int32_t *length, int32_t *gapopen,
                   int32_t *mismatch, double *identity, cudaStream_t st) {
    if (n <= 0) return TPZ_OK;
    int64_t *qoff = nullptr, *soff = nullptr;
    int32_t *valid = nullptr;
    auto cleanup = [&]() {
        for (void *p : {(void *)qoff, (void *)soff, (void *)valid}) if (p) cudaFreeAsync(p, st);
    };
    if (cudaMallocAsync((void **)&qoff, 8 * n, st) || cudaMallocAsync((void **)&soff, 8 * n, st) ||
        cudaMallocAsync((void **)&valid, 4 * n, st)) {
        cleanup();
        return cuda_fail(cudaGetLastError(), "reported_stats");
    }
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096));
    reported_pairs_kernel<<<grid, 256, 0, st>>>(n, query_of, qoff_q, pstart, protein, sw_status,
                                                qoff, soff, valid, qstart, sstart, length, gapopen,
                                                mismatch, identity);
    PairArgs a;
    memset(&a, 0, sizeof a);
    a.n = n; a.q = qtext; a.s = T; a.qoff = qoff; a.soff = soff;
    a.read_end = qend; a.ref_end = send; a.score = raw; a.valid = valid;
    memcpy(a.mat, mat, 625);
    memcpy(a.xmap, xmap, 128);
    a.translate = 1;
    int mn = 0;
    for (int i = 0; i < 625; ++i) mn = std::min<int>(mn, mat[i]);
    a.bias = -mn;
    a.gap_open = go; a.gap_extend = ge;
    a.qstart = qstart; a.sstart = sstart; a.length = length; a.gapopen = gapopen;
    a.mismatch = mismatch; a.identity = identity;
    const int rc = stats_batch(a, st);
    cleanup();
    return rc;
}

}  // namespace stats
}  // namespace tpz

extern "C" int tpz_sw_stats_device(int64_t n, const int8_t *q, const int64_t *qoff,
                                   const int32_t *qlen, const int8_t *s, const int64_t *soff,
                                   const int32_t *slen, const int8_t *mat625_host, int gap_open,
                                   int gap_extend, const int32_t *read_end, const int32_t *ref_end,
                                   const int32_t *score, int32_t *qstart, int32_t *sstart,
                                   int32_t *length, int32_t *gapopen, int32_t *mismatch,
                                   double *identity, void *stream) {
    if (n < 0 || !mat625_host) {
        tpz::set_error("tpz_sw_stats_device: n < 0 or NULL matrix");
        return TPZ_E_ARG;
    }
    if (n == 0) return TPZ_OK;
    if (!q || !qoff || !qlen || !s || !soff || !slen || !read_end || !ref_end || !score ||
        !qstart || !sstart || !length || !gapopen || !mismatch || !identity) {
        tpz::set_error("tpz_sw_stats_device: NULL buffer");
        return TPZ_E_ARG;
    }
    tpz::stats::PairArgs a;
    memset(&a, 0, sizeof a);
    a.n = n; a.q = q; a.qoff = qoff; a.qlen = qlen; a.s = s; a.soff = soff; a.slen = slen;
    a.read_end = read_end; a.ref_end = ref_end; a.score = score;
    memcpy(a.mat, mat625_host, 625);
    int mn = 0;
    for (int i = 0; i < 625; ++i) mn = std::min<int>(mn, mat625_host[i]);
    a.bias = -mn;
    a.gap_open = gap_open; a.gap_extend = gap_extend;
    a.qstart = qstart; a.sstart = sstart; a.length = length; a.gapopen = gapopen;
    a.mismatch = mismatch; a.identity = identity;
    return tpz::stats::stats_batch(a, (cudaStream_t)stream);
}
