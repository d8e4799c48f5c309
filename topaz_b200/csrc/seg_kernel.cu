// seg_kernel.cu -- query ingest on the device: SEG low-complexity masking
// (run_seg, src/seg_wrapper.c:15-49 over src/seg/seg.c:147-408 and
// src/seg/genwin.c:170-323: window 12, trigger complexity 2.2, extension
// 2.5, maximal trim 100, hard mask 'X'), then the internal alphabet
// (seq_2internal, src/seq.c:106-117) -- what run_query does to each query
// before seeding (src/engine.c:250-277).
//
// One thread per query.  SEG (Wootton & Federhen 1993) decides with doubles;
// for the masks to equal the host's bit for bit, every transcendental value
// comes from tables the host computes with the C library (the full-window
// entropy terms, log(x / t) of the partial-window terms, ln n! rounded to 6
// decimals), and the device only adds, subtracts, multiplies and divides,
// in the host's order, rounded to nearest without fused multiply-adds (this
// file is compiled with -fmad=false).
//
// The per-query state: a window's residue counts and the descending
// multiset of its non-zero counts (the entropy and the probability depend
// only on that multiset), the entropy of every 12-residue window, and a
// stack of nested searches (a trigger window lost to a segment's left trim
// is searched again in the part that was cut, which is at most 100 residues
// long, so nesting stays shallow).  Segments merge as they are found: an
// overlapping successor gives its end to the segment before it.
#include <algorithm>
#include <mutex>

#include "tpz_common.cuh"

extern "C" void tpzh_seg_tables(double *ent_full, double *logxr, double *lnfac_out, int n);
extern "C" char tpzh_aa2internal(char c);

namespace tpz {
namespace seg {

constexpr int kWin = 12;
constexpr int kDown = (kWin + 1) / 2 - 1;     // 5
constexpr int kUp = kWin - kDown;             // 7
constexpr int kMaxTrim = 100;
constexpr double kLoCut = 2.2, kHiCut = 2.5;
constexpr double kLn2 = 0.69314718055994530941723212145818;
constexpr double kLn20 = 2.9957322735539909;
constexpr int kLnFac = 10001;                 // ln n! entries (queries are shorter)
constexpr int kScratchExtra = 1024;           // entropy slots beyond the query, for nested searches
constexpr int kMaxDepth = 24;

struct Tables {
    double ent_full[kWin + 1];
    double logxr[(kWin + 1) * (kWin + 1)];
    int8_t res_index[256];        // residue -> 0..19, -1 not counted
    char to_internal[256];
};

struct Args {
    const char *in;
    char *out;
    const int64_t *off;
    const int32_t *len;
    int64_t n;
    int seg;
    double *scratch;              // per query at off[i] + kScratchExtra * i
    const double *lnfac;
    int *err;                     // set when a query needed more scratch than it has
};

struct Win {
    int start, len;
    int comp[20];
    int sv[21];                   // descending non-zero counts, 0-terminated
};

__device__ void win_open(const char *s, const Tables &t, int start, int len, Win &w) {
    w.start = start; w.len = len;
    for (int k = 0; k < 20; ++k) w.comp[k] = 0;
    for (int i = start; i < start + len; ++i) {
        const int k = t.res_index[(uint8_t)s[i]];
        if (k >= 0) w.comp[k]++;
    }
    int n = 0;
    for (int k = 0; k < 20; ++k) if (w.comp[k]) w.sv[n++] = w.comp[k];
    for (int k = n; k < 21; ++k) w.sv[k] = 0;
    for (int a = 1; a < n; ++a) {               // descending order
        const int v = w.sv[a];
        int b = a - 1;
        while (b >= 0 && w.sv[b] < v) { w.sv[b + 1] = w.sv[b]; --b; }
        w.sv[b + 1] = v;
    }
}

// the class of count c shrinks by one: its last entry
__device__ __forceinline__ void sv_dec(int *sv, int c) {
    for (int i = 0; sv[i] != 0; ++i)
        if (sv[i] == c && sv[i + 1] < c) { sv[i] = c - 1; return; }
}

// the class of count c grows by one: its first entry (c = 0: the terminator)
__device__ __forceinline__ void sv_inc(int *sv, int c) {
    int i = 0;
    while (sv[i] != c) ++i;
    sv[i]++;
}

// one residue to the right inside [.., end); false when it would leave
__device__ bool win_shift(const char *s, const Tables &t, int end, Win &w) {
    if (w.start + 1 + w.len > end) return false;
    const int out = t.res_index[(uint8_t)s[w.start]];
    const int in = t.res_index[(uint8_t)s[w.start + w.len]];
    w.start++;
    if (out >= 0) sv_dec(w.sv, w.comp[out]--);
    if (in >= 0) sv_inc(w.sv, w.comp[in]++);
    return true;
}

__device__ double sv_entropy(const Tables &t, const int *sv) {
    int total = 0, n = 0;
    while (sv[n] != 0) total += sv[n++];
    double ent = 0.0;
    if (total == kWin) {
        for (int i = 0; i < n; ++i) ent += t.ent_full[sv[i]];
        return ent;
    }
    if (total == 0) return 0.;
    const double rt = 1. / (double)total;
    for (int i = 0; i < n; ++i) {
        const double x = sv[i];
        ent += x * t.logxr[total * (kWin + 1) + sv[i]];
    }
    return -ent * rt / kLn2;
}

// ln of the number of ways 20 residue types take the multiset's counts
__device__ double sv_lnass(const double *lnfac, const int *sv) {
    double ans = lnfac[20];
    if (sv[0] == 0) return ans;
    int total = 20, cls = 1, prev = sv[0], i = 0;
    const int *p = sv;
    for (;;) {
        if (++i == 20) { ans -= lnfac[cls]; break; }
        const int cur = *++p;
        if (cur == prev) { cls++; continue; }
        total -= cls;
        ans -= lnfac[cls];
        if (cur == 0) { ans -= lnfac[total]; break; }
        cls = 1;
        prev = cur;
    }
    return ans;
}

__device__ double sv_lnperm(const double *lnfac, const int *sv, int tot) {
    double ans = lnfac[tot];
    for (int i = 0; sv[i] != 0; ++i) ans -= lnfac[sv[i]];
    return ans;
}

__device__ double sv_prob(const double *lnfac, const int *sv, int total) {
    const double totseq = ((double)total) * kLn20;
    return sv_lnass(lnfac, sv) + sv_lnperm(lnfac, sv, total) - totseq;
}

// the most improbable sub-window of s[start, start + len) at least
// len - 100 long: moves *left / *right to its ends
__device__ void seg_trim(const char *s, const Tables &t, const double *lnfac, int start, int len,
                         int *left, int *right) {
    int lend = 0, rend = len - 1, minlen = 1;
    if (len - kMaxTrim > minlen) minlen = len - kMaxTrim;
    double minprob = 1.;
    for (int wl = len; wl > minlen; --wl) {
        Win w;
        win_open(s, t, start, wl, w);
        int i = 0;
        for (;;) {
            const double p = sv_prob(lnfac, w.sv, wl);
            if (p < minprob) { minprob = p; lend = i; rend = wl + i - 1; }
            if (!win_shift(s, t, start + len, w)) break;
            ++i;
        }
    }
    *left += lend;
    *right -= (len - rend - 1);
}

struct Frame {
    int start, len;               // the searched part of the query
    int i, lowlim, last;          // loop state
    int hoff;                     // entropies at scratch + hoff
    int pend_left, pend_right, pend_hii;   // a segment waiting for its nested search
    bool resume;
};

struct Merger {                   // mergesegs, as segments arrive
    int cb = 0, ce = -1;
    bool open = false;
    __device__ void flush(char *o) {
        if (open) for (int k = cb; k <= ce; ++k) o[k] = 'X';
        open = false;
    }
    __device__ void push(char *o, int b, int e) {
        if (open && ce >= b) { ce = e; return; }
        flush(o);
        cb = b; ce = e; open = true;
    }
};

__global__ void prepare_kernel(const __grid_constant__ Tables t, Args a) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < a.n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const char *s = a.in + a.off[q];
        char *o = a.out + a.off[q];
        const int len = a.len[q];
        for (int i = 0; i < len; ++i) o[i] = s[i];
        if (a.seg && len >= kLnFac) {
            atomicExch(a.err, 2);                 // beyond the ln n! table
        } else if (a.seg && len >= kWin) {
            double *H = a.scratch + a.off[q] + kScratchExtra * q;
            const int cap = len + kScratchExtra;
            Merger mg;
            Frame st[kMaxDepth];
            int top = 0;
            auto open_frame = [&](Frame &f, int start, int flen, int hoff) -> bool {
                f.start = start; f.len = flen; f.hoff = hoff; f.resume = false;
                if (kWin > flen) { f.i = 1; f.last = 0; return true; }
                if (hoff + flen > cap) return false;
                double *h = H + hoff;
                for (int i = 0; i < flen; ++i) h[i] = -1.;
                const int first = kDown;
                f.last = flen - kUp;
                Win w;
                win_open(s, t, start, kWin, w);
                for (int i = first; i <= f.last; ++i) {
                    h[i] = sv_entropy(t, w.sv);
                    win_shift(s, t, start + flen, w);
                }
                f.i = first;
                f.lowlim = first;
                return true;
            };
            bool ok = open_frame(st[0], 0, len, 0);
            while (ok && top >= 0) {
                Frame &f = st[top];
                const double *h = H + f.hoff;
                if (f.resume) {
                    // the nested search is done: this segment, then go on
                    f.resume = false;
                    mg.push(o, f.pend_left + f.start, f.pend_right + f.start);
                    const int ni = f.pend_hii < f.pend_right + kDown ? f.pend_hii : f.pend_right + kDown;
                    f.lowlim = ni + 1;
                    f.i = ni + 1;
                }
                bool nested = false;
                for (; f.i <= f.last; ++f.i) {
                    const int i = f.i;
                    if (!(h[i] <= kLoCut && h[i] != -1)) continue;
                    int j;
                    for (j = i; j >= f.lowlim; --j) if (h[j] == -1 || h[j] > kHiCut) break;
                    const int loi = j + 1;
                    for (j = i; j <= f.last; ++j) if (h[j] == -1 || h[j] > kHiCut) break;
                    const int hii = j - 1;
                    int leftend = loi - kDown;
                    int rightend = hii + kUp - 1;
                    seg_trim(s, t, a.lnfac, f.start + leftend, rightend - leftend + 1, &leftend,
                             &rightend);
                    if (i + kUp - 1 < leftend) {
                        // the trigger window fell to the left trim: search the cut part first
                        const int lend = loi - kDown, rend = leftend - 1;
                        f.pend_left = leftend; f.pend_right = rightend; f.pend_hii = hii;
                        f.resume = true;
                        if (top + 1 >= kMaxDepth) { ok = false; break; }
                        ok = open_frame(st[top + 1], f.start + lend, rend - lend + 1, f.hoff + f.len);
                        ++top;
                        nested = true;
                        break;
                    }
                    mg.push(o, leftend + f.start, rightend + f.start);
                    f.i = hii < rightend + kDown ? hii : rightend + kDown;
                    f.lowlim = f.i + 1;
                }
                if (!nested && ok) --top;
            }
            if (!ok) atomicExch(a.err, 1);
            mg.flush(o);
        }
        for (int i = 0; i < len; ++i) o[i] = t.to_internal[(uint8_t)o[i]];
    }
}

static Tables g_tables;
static double *g_lnfac_host = nullptr;

static void host_tables() {
    if (g_lnfac_host) return;
    static double ln[kLnFac];
    tpzh_seg_tables(g_tables.ent_full, g_tables.logxr, ln, kLnFac);
    const char *aa = "ACDEFGHIKLMNPQRSTVWY";
    for (int i = 0; i < 256; ++i) g_tables.res_index[i] = -1;
    for (int i = 0; aa[i]; ++i) {
        g_tables.res_index[(uint8_t)aa[i]] = (int8_t)i;
        g_tables.res_index[(uint8_t)(aa[i] + 32)] = (int8_t)i;
    }
    for (int c = 0; c < 256; ++c) g_tables.to_internal[c] = tpzh_aa2internal((char)c);
    g_lnfac_host = ln;
}

// SEG (seg != 0) + internal alphabet of queries in[off[i] .. + len[i]) into
// out (same offsets; in and out must not overlap); queries are disjoint.
int prepare_device(const char *in, char *out, const int64_t *off, const int32_t *len, int64_t n,
                   int64_t total_bytes, int seg, cudaStream_t st) {
    if (n <= 0) return TPZ_OK;
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> lk(mu);
        host_tables();
    }
    double *lnfac = nullptr, *scratch = nullptr;
    int *err = nullptr;
    auto cleanup = [&]() {
        for (void *p : {(void *)lnfac, (void *)scratch, (void *)err}) if (p) cudaFreeAsync(p, st);
    };
    const size_t sbytes = seg ? sizeof(double) * ((size_t)total_bytes + (size_t)kScratchExtra * n) : 16;
    if (cudaMallocAsync((void **)&lnfac, sizeof(double) * kLnFac, st) ||
        cudaMallocAsync((void **)&scratch, sbytes, st) || cudaMallocAsync((void **)&err, 4, st)) {
        cleanup();
        return cuda_fail(cudaGetLastError(), "prepare_device");
    }
    int herr = 0;
    if (cudaMemcpyAsync(lnfac, g_lnfac_host, sizeof(double) * kLnFac, cudaMemcpyHostToDevice, st) ||
        cudaMemsetAsync(err, 0, 4, st)) {
        cleanup();
        return cuda_fail(cudaGetLastError(), "prepare_device copies");
    }
    Args a;
    a.in = in; a.out = out; a.off = off; a.len = len; a.n = n; a.seg = seg;
    a.scratch = scratch; a.lnfac = lnfac; a.err = err;
    // few long-running threads: small blocks spread them over the SMs
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 31) / 32, 8192));
    prepare_kernel<<<grid, 32, 0, st>>>(g_tables, a);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st) || cudaStreamSynchronize(st)) {
        cleanup();
        return cuda_fail(cudaGetLastError(), "prepare_kernel");
    }
    cleanup();
    if (herr == 2) {
        set_error("query ingest: SEG on the device takes queries of at most 10000 residues");
        return TPZ_E_RANGE;
    }
    if (herr) {
        set_error("query ingest: SEG needed more nested searches than the device keeps");
        return TPZ_E_DEVICE;
    }
    return TPZ_OK;
}

}  // namespace seg
}  // namespace tpz

extern "C" int tpz_prepare_queries_device(char *cat, const int64_t *off, const int32_t *len,
                                          int64_t n, int64_t total_bytes, int seg, void *stream) {
    if (n < 0 || total_bytes < 0 || (n > 0 && (!cat || !off || !len))) {
        tpz::set_error("tpz_prepare_queries_device: bad arguments");
        return TPZ_E_ARG;
    }
    if (n == 0) return TPZ_OK;
    cudaStream_t st = (cudaStream_t)stream;
    char *in = nullptr;
    if (cudaMallocAsync((void **)&in, std::max<int64_t>(total_bytes, 1), st) != cudaSuccess)
        return tpz::cuda_fail(cudaGetLastError(), "tpz_prepare_queries_device");
    int rc = TPZ_OK;
    if (cudaMemcpyAsync(in, cat, total_bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        rc = tpz::cuda_fail(cudaGetLastError(), "tpz_prepare_queries_device copy");
    if (rc == TPZ_OK) rc = tpz::seg::prepare_device(in, cat, off, len, n, total_bytes, seg, st);
    cudaFreeAsync(in, st);
    return rc;
}
