// bm_select.cuh -- pair combine and move selection of the sweep.
//
// k_combine64: 64x64 tiles of the upper triangle of S.  Each tile (I,J), I<=J,
//   reads S[I][J] and S[J][I] once (coalesced rows), forms
//   delta(a,b) = S[a][b] + S[b][a] - S[a][a] - S[b][b] and writes, for every
//   vertex of the tile, its best partner inside the tile to a partial array
//   P[tile column][vertex]; k_best_reduce folds the partials into rowbest.
//   No atomics; every (tile, vertex) slot is written exactly once.
// k_commit_group: the sequential set commit (candidates sorted by delta desc,
//   skip a pair whose vertex already moved, re-evaluate it on the current
//   matching, commit iff > 0), several pairs per step.
#pragma once
#include <climits>
#include "bm_kernels.cuh"

namespace bm {

constexpr int kTile = 64;

// One TxT tile (ti <= tj) of the upper triangle, 256 threads (T = 32 or 64).
// Shared memory of one combine tile pass.
template <int T> struct CombineSmem {
    int sA[T][T + 1];               // sA[r][c] = S[a0+r][b0+c]
    int sB[T][T + 1];               // sB[r][c] = S[b0+r][a0+c]
    int dA[T], dB[T];
    unsigned long long cpart[8][T];
};

// One tile pair by 256 threads (tid 0..255 among them; `sync` is a barrier
// over exactly those threads), staged in `sm`.
template <int T, typename Sync>
__device__ __forceinline__ void combine_tile_on(const int* __restrict__ S, int n, int ti, int tj,
                                                unsigned long long* __restrict__ part, int* __restrict__ all_out,
                                                CombineSmem<T>& sm, int tid, Sync sync) {
    constexpr int CL = T / 32;            // columns per lane
    const int a0 = ti * T, b0 = tj * T;
    const int lane = tid & 31, wid = tid >> 5;  // 8 warps
    if ((n & 3) == 0) {
        // 16-byte streaming loads: with n a multiple of 4 every 4-column group
        // of a row is aligned and lies wholly inside or outside the matrix
        for (int i = tid; i < T * T / 4; i += 256) {
            const int r = i / (T / 4), c = (i % (T / 4)) * 4;
            const int a = a0 + r, b = b0 + c;
            const int bb = b0 + r, aa = a0 + c;
            int4 va = make_int4(0, 0, 0, 0), vb = make_int4(0, 0, 0, 0);
            if (a < n && b < n) va = __ldcs(reinterpret_cast<const int4*>(S + (size_t)a * n + b));
            if (bb < n && aa < n) vb = __ldcs(reinterpret_cast<const int4*>(S + (size_t)bb * n + aa));
            sm.sA[r][c] = va.x; sm.sA[r][c + 1] = va.y; sm.sA[r][c + 2] = va.z; sm.sA[r][c + 3] = va.w;
            sm.sB[r][c] = vb.x; sm.sB[r][c + 1] = vb.y; sm.sB[r][c + 2] = vb.z; sm.sB[r][c + 3] = vb.w;
        }
    } else {
        for (int i = tid; i < T * T; i += 256) {
            const int r = i / T, c = i % T;
            const int a = a0 + r, b = b0 + c;
            sm.sA[r][c] = (a < n && b < n) ? S[(size_t)a * n + b] : 0;
            const int bb = b0 + r, aa = a0 + c;
            sm.sB[r][c] = (bb < n && aa < n) ? S[(size_t)bb * n + aa] : 0;
        }
    }
    if (tid < T) {
        const int a = a0 + tid, b = b0 + tid;
        sm.dA[tid] = a < n ? S[(size_t)a * n + a] : 0;
        sm.dB[tid] = b < n ? S[(size_t)b * n + b] : 0;
    }
    sync();
    const bool diag = (ti == tj);
    // bests as 32-bit (delta, partner) pairs -- larger delta, then smaller
    // partner -- packed into the 64-bit key only for the reductions
    int cbd[CL], cbi[CL];
#pragma unroll
    for (int q = 0; q < CL; q++) { cbd[q] = INT_MIN; cbi[q] = INT_MAX; }
    for (int r = wid; r < T; r += 8) {
        const int a = a0 + r;
        int rd = INT_MIN, ri = INT_MAX;
        if (a < n) {
#pragma unroll
            for (int q = 0; q < CL; q++) {
                const int c = lane + 32 * q, b = b0 + c;
                if (b < n && b != a) {
                    const int d = sm.sA[r][c] + sm.sB[c][r] - sm.dA[r] - sm.dB[c];
                    if (d > rd || (d == rd && b < ri)) { rd = d; ri = b; }
                    if (d > cbd[q] || (d == cbd[q] && a < cbi[q])) { cbd[q] = d; cbi[q] = a; }
                    if (all_out && a < b) all_out[(long long)a * (2LL * n - a - 1) / 2 + (b - a - 1)] = d;
                }
            }
        }
        unsigned long long rb = ri == INT_MAX ? 0ull : pack_best(rd, ri);
        for (int o = 16; o; o >>= 1) rb = kmax(rb, __shfl_xor_sync(0xffffffffu, rb, o));
        if (lane == 0 && a < n) part[(size_t)tj * n + a] = rb;  // row partial of a over this tile
    }
    unsigned long long cb[CL];
#pragma unroll
    for (int q = 0; q < CL; q++) cb[q] = cbi[q] == INT_MAX ? 0ull : pack_best(cbd[q], cbi[q]);
    // column partials (vertices b of the tile, over this tile's rows); a
    // diagonal tile's row partials already cover both orders of every pair
    if (!diag) {
#pragma unroll
        for (int q = 0; q < CL; q++) sm.cpart[wid][lane + 32 * q] = cb[q];
        sync();
        if (tid < T) {
            unsigned long long k = sm.cpart[0][tid];
            for (int w = 1; w < 8; w++) k = kmax(k, sm.cpart[w][tid]);
            const int b = b0 + tid;
            if (b < n) part[(size_t)ti * n + b] = k;
        }
    }
}

// One tile pair by a 256-thread block.
template <int T>
__device__ __forceinline__ void combine_tile(const int* __restrict__ S, int n, int ti, int tj,
                                             unsigned long long* __restrict__ part, int* __restrict__ all_out) {
    __shared__ CombineSmem<T> sm;
    combine_tile_on<T>(S, n, ti, tj, part, all_out, sm, threadIdx.x, [] { __syncthreads(); });
}

static __global__ void __launch_bounds__(256)
k_combine64(const int* __restrict__ S, int n, unsigned long long* __restrict__ part,
            int* __restrict__ all_out) {
    const int ti = blockIdx.y, tj = blockIdx.x;
    if (ti > tj) return;
    combine_tile<kTile>(S, n, ti, tj, part, all_out);
}

// rowbest[x] = max over tile columns t of part[t][x]
static __global__ void k_best_reduce(const unsigned long long* __restrict__ part, int n, int tiles,
                              unsigned long long* __restrict__ rowbest) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    unsigned long long k = 0;
    for (int t = 0; t < tiles; t++) k = kmax(k, part[(size_t)t * n + x]);
    rowbest[x] = k;
}

// ---------------------------------------------------------------------------
// Set commit (one CTA).  The rule is sequential over the sorted candidates:
//   * skip the pair if either vertex already moved in this sweep;
//   * otherwise its current delta is the sweep delta plus, for every G1 edge
//     from one of its vertices x to an already-moved vertex z, the change of
//     that edge's term between z's pre-move image (pold) and its image now;
//     a pair with at least one moved neighbour is the "re-verified" case
//     (counted, and limited by max_verify);
//   * commit iff the current delta is > 0.
// It is executed CG pairs at a time: the CTA makes one coalesced pass over
// the step's edge lists (entries spread evenly over all threads, so a hub
// pair does not stall the step), accumulating each pair's correction
// from moved neighbours (a flag check per entry; W2 is read only for moved
// neighbours) and noting which earlier pairs of the step it shares a vertex
// with or is G1-adjacent to.  For an entry whose neighbour belongs to an
// earlier pair i of the step, the scan also adds the change that pair i's
// swap would make to this pair's delta into cc[j][i] (each G1 edge has one
// endpoint outside the pair, so these changes add up).  Warp 0 then decides
// the pairs in order: a pair sharing a vertex with an earlier committed pair
// is skipped, a pair next to a moved vertex (an earlier step's, or an earlier
// committed pair of this step) is re-verified as its sweep delta plus those
// changes, and it commits iff that is > 0.  A pair's delta depends only on p
// at its vertices and their G1 neighbours, so every decision equals the
// one-at-a-time rule's, re-verification budget included, and no pair is
// scanned twice.
constexpr int kCG = 16;                // pairs per step of the cluster commit (16-bit vertex marks)
constexpr int kCGWide = 32;            // ... when 32-bit marks fit in shared memory
constexpr int kCGBatch = 8;            // pairs per step of a one-CTA commit (batched instances)

// 16-bit atomic OR in shared memory through the aligned 32-bit word.
__device__ __forceinline__ void atomicOr_u16(uint16_t* p, uint16_t v) {
    const size_t addr = reinterpret_cast<size_t>(p);
    unsigned* w = reinterpret_cast<unsigned*>(addr & ~(size_t)3);
    atomicOr(w, (unsigned)v << ((addr & 2) ? 16 : 0));
}

// Several CTAs on one set commit, as one thread-block cluster: every CTA keeps
// the same shared state and makes the same gather and the same ordered
// decisions; only the step's list scan is divided.  Each CTA publishes its
// per-pair partial sums in its own shared memory (two buffers, by step
// parity), arrives on every CTA's step mbarrier, waits on its own (bounded),
// and reads the others' partials through distributed shared memory.
struct CommitGrid {
    int nct;          // CTAs of the cluster (1: a single CTA, no exchange)
    int* err;         // bit 1 set when a cluster wait runs out
    int stall = 0;    // test hook (bm_test_stall): no CTA arrives in the first exchange
};

__device__ __forceinline__ uint32_t cluster_map(uint32_t local_addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(rank));
    return r;
}

// Arrive on the step mbarrier of every CTA of the cluster, then wait (bounded)
// for this CTA's to complete the phase; false on timeout.  Thread 0 of each
// CTA does the arrivals and the wait; the CTA syncs around it.
//
// A CTA whose wait runs out stays resident for one more full wait window
// before it reports the timeout (and the caller leaves): a peer whose own wait
// completed just then still reads this CTA's partial sums and arrives on its
// mbarrier at the next step, and both must reach a CTA that has not exited.
// That peer then times out at the next step in turn, so every CTA stops
// within two steps.  `stall` (the test hook) skips this CTA's arrivals and
// shortens both windows: when every CTA stalls, every wait runs out at the
// same step and no CTA touches another's shared memory afterwards.
__device__ __forceinline__ bool cluster_step_sync(uint32_t bar, uint32_t phase, int nct, int* err, bool stall = false) {
    __shared__ int s_cok;
    __syncthreads();
    if (!stall && threadIdx.x < (unsigned)nct) {  // thread r arrives on CTA r's mbarrier
        const uint32_t rb = cluster_map(bar, threadIdx.x);
        asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" :: "r"(rb) : "memory");
    }
    if (threadIdx.x == 0) {
        const int limit = stall ? (1 << 12) : (1 << 22);
        int ok = 0;
        for (int it = 0; it < limit; it++) {
            uint32_t done;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done) : "r"(bar), "r"(phase) : "memory");
            if (done) { ok = 1; break; }
        }
        if (!ok) {
            // the linger window: as many polls again, whatever they return
            // (a poll suspends while the phase is open and returns at once
            // after it completes, so this lasts at least milliseconds)
            for (int it = 0; it < limit; it++)
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%0], %1;\n\t}"
                    :: "r"(bar), "r"(phase) : "memory");
            atomicOr(err, 2);
        }
        s_cok = ok;
    }
    __syncthreads();
    return s_cok != 0;
}

// The set commit of one instance; all 1024 threads of the block call it.
// smem: commit_group_smem(n) bytes of dynamic shared memory.
// Per-vertex step marks: bit i = the vertex belongs to pair i of the step.
template <int CG> struct MarkOf { typedef uint16_t T; };
template <> struct MarkOf<32> { typedef uint32_t T; };

template <bool W16, int CG = kCG>
__device__ __forceinline__ void commit_group(const DevView<W16>& g, const unsigned long long* __restrict__ keys,
                                             int lim, int max_verify, CommitStats* __restrict__ st,
                                             unsigned char* smem, const int4* __restrict__ cinfo = nullptr,
                                             CommitGrid grid = CommitGrid{1, nullptr}) {
    typedef Ent<W16> EN;
    // shared: used[n] flags, then the matching and the pre-move images as
    // 16-bit ids (n <= 65535, so the "unmatched" value n fits)
    const int n = g.n;
    unsigned char* used = smem;
    uint16_t* p16 = reinterpret_cast<uint16_t*>(smem + ((n + 15) & ~15));
    uint16_t* q16 = p16 + ((n + 8) & ~7);
    typedef typename MarkOf<CG>::T MarkT;
    MarkT* mark = reinterpret_cast<MarkT*>(q16 + ((n + 8) & ~7));  // bit i set: vertex belongs to pair i of the step
    __shared__ int s_lo[CG], s_hi[CG], s_d0[CG];
    __shared__ int s_corr[CG], s_cnt[CG], s_pre[CG + 1];
    __shared__ unsigned s_imask[CG];   // earlier pairs of the step G1-adjacent to this one
    __shared__ unsigned s_share[CG];   // earlier pairs of the step sharing a vertex with this one
    __shared__ unsigned s_dead;         // pairs with a vertex already moved when the step starts
    __shared__ int s_inf[CG][8];       // la0, la, ia0, ia, lb0, lb, ib0, ib
    __shared__ int s_segpre[4 * CG + 1];  // the step's lists as segments 4j + k: prefix of their lengths
    __shared__ int s_segoff[4 * CG];      // first entry of segment 4j + k in ent1o (k even) or ent1i (k odd)
    __shared__ int s_n, s_k, s_scanned;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nct = grid.nct;
    int ct = 0;
    if (nct > 1) asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(ct));
    int gstep = 0;      // steps taken, the same in every CTA
    bool aborted = false;
    __shared__ __align__(8) unsigned long long s_cbar;   // the step mbarrier (nct arrivals per phase)
    constexpr int kPart = (3 + CG + 3) & ~3;            // a pair's partials, padded to whole 16-byte words
    __shared__ __align__(16) int s_cpart[2][CG][kPart];  // this CTA's partial sums, by step parity
    __shared__ int s_cc[CG][CG];   // s_cc[j][i]: change of pair j's delta if earlier pair i commits
    const uint32_t cbar = (uint32_t)__cvta_generic_to_shared(&s_cbar);
    if (nct > 1) {
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(cbar), "r"(nct) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        // every CTA's mbarrier is initialised before anyone arrives on it
        asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
        asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
    for (int i = tid; i < n; i += blockDim.x) { used[i] = 0; p16[i] = (uint16_t)g.p[i]; mark[i] = 0; }
    for (int i = tid; i < CG * CG; i += blockDim.x) (&s_cc[0][0])[i] = 0;
    if (tid == 0) { s_n = 0; s_k = 0; s_scanned = 0; p16[n] = (uint16_t)n; }
    long long total = 0, entries = 0;
    int verified = 0, committed = 0, steps = 0;
    // warp 0: the next kPF candidates (keys and list extents), prefetched into
    // shared memory at the end of each step; a step scans ~180 candidates early
    // in a descent, so a 32-wide window left one L2 round trip per further 32
    constexpr int kPF = 256;
    int pf_base = -1;                  // warp 0: first candidate of the prefetched window
    bool pf_waited = false;
    __shared__ unsigned long long s_pfkey[kPF];
    __shared__ int4 s_pfinf[kPF][2];
    __syncthreads();
    for (;;) {
        // ---- warp 0: the next live candidates, then the
        //      per-pair list extents and their prefix (lane j = pair j) ----
        if (wid == 0) {
            int cnt = s_n, k = s_k, scanned = s_scanned;
            while (cnt < CG && k < lim) {
                const int idx = k + lane;
                unsigned long long key;
                int4 i0 = make_int4(0, 0, 0, 0), i1 = make_int4(0, 0, 0, 0);
                const int off = k - pf_base;
                if (cinfo && pf_base >= 0 && off >= 0 && off + 32 <= kPF) {   // inside the prefetched window
                    if (!pf_waited) {   // every lane's copies have landed (lanes read each other's slots)
                        asm volatile("cp.async.wait_group 0;" ::: "memory");
                        __syncwarp();
                        pf_waited = true;
                    }
                    key = s_pfkey[off + lane]; i0 = s_pfinf[off + lane][0]; i1 = s_pfinf[off + lane][1];
                } else {
                    key = idx < lim ? keys[idx] : ~0ull;
                    if (cinfo && idx < lim) { i0 = cinfo[2 * idx]; i1 = cinfo[2 * idx + 1]; }
                }
                const bool valid = key != ~0ull;
                const int lo = valid ? (int)((key >> 16) & 0xffffu) : 0;
                const int hi = valid ? (int)(key & 0xffffu) : 0;
                const bool live = valid && !used[lo] && !used[hi];
                const unsigned vmask = __ballot_sync(0xffffffffu, valid);
                const unsigned lmask = __ballot_sync(0xffffffffu, live);
                const int room = CG - cnt;
                const int before = __popc(lmask & ((1u << lane) - 1u));
                const int nvalid = __popc(vmask);  // valid keys form a prefix
                int consumed = nvalid, took = __popc(lmask);
                if (took > room) {  // stop just before the (room+1)-th live candidate
                    const unsigned over = __ballot_sync(0xffffffffu, live && before == room);
                    consumed = __ffs(over) - 1;
                    took = room;
                }
                if (live && before < room) {
                    const int q = cnt + before;
                    s_lo[q] = lo; s_hi[q] = hi;
                    s_d0[q] = (int)(0x7fffffffu - (unsigned)(key >> 32));
                    if (!cinfo) {  // list extents straight from the offsets
                        i0.x = g.off1o[lo]; i0.y = g.off1o[lo + 1] - i0.x;
                        i0.z = g.off1i[lo]; i0.w = g.off1i[lo + 1] - i0.z;
                        i1.x = g.off1o[hi]; i1.y = g.off1o[hi + 1] - i1.x;
                        i1.z = g.off1i[hi]; i1.w = g.off1i[hi + 1] - i1.z;
                    }
                    s_inf[q][0] = i0.x; s_inf[q][1] = i0.y; s_inf[q][2] = i0.z; s_inf[q][3] = i0.w;
                    s_inf[q][4] = i1.x; s_inf[q][5] = i1.y; s_inf[q][6] = i1.z; s_inf[q][7] = i1.w;
                }
                cnt += took;
                k += consumed;
                scanned += consumed;
                if (consumed == nvalid && nvalid < 32) { k = lim; break; }
            }
            // prefetch the next window (its keys and list extents); it is used as
            // is, since only the used flags change and those are read at use
            if (cinfo) {  // asynchronous copies straight into shared memory, lane l the slots l, l + 32, ...
                if (!pf_waited && pf_base >= 0) {   // copies of a window never read must land first
                    asm volatile("cp.async.wait_group 0;" ::: "memory");
                }
                __syncwarp();   // every lane is done reading the previous window
                pf_base = k;
                pf_waited = false;
                for (int h = 0; h < kPF / 32; h++) {
                    const int slot = 32 * h + lane, idx = k + slot;
                    if (idx < lim) {
                        const uint32_t dk = (uint32_t)__cvta_generic_to_shared(&s_pfkey[slot]);
                        const uint32_t di = (uint32_t)__cvta_generic_to_shared(&s_pfinf[slot][0]);
                        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(dk), "l"(keys + idx) : "memory");
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(di), "l"(cinfo + 2 * idx) : "memory");
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(di + 16), "l"(cinfo + 2 * idx + 1) : "memory");
                    } else {
                        s_pfkey[slot] = ~0ull;
                        s_pfinf[slot][0] = make_int4(0, 0, 0, 0);
                        s_pfinf[slot][1] = make_int4(0, 0, 0, 0);
                    }
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
            }
            __syncwarp();
            int len = 0;
            if (lane < cnt) {
                const int a = s_lo[lane], b = s_hi[lane];
                len = s_inf[lane][1] + s_inf[lane][3] + s_inf[lane][5] + s_inf[lane][7];
                s_corr[lane] = 0; s_cnt[lane] = 0; s_imask[lane] = 0;
                if (sizeof(MarkT) == 2) {
                    atomicOr_u16(reinterpret_cast<uint16_t*>(&mark[a]), (uint16_t)(1u << lane));
                    atomicOr_u16(reinterpret_cast<uint16_t*>(&mark[b]), (uint16_t)(1u << lane));
                } else {
                    atomicOr(reinterpret_cast<unsigned*>(&mark[a]), 1u << lane);
                    atomicOr(reinterpret_cast<unsigned*>(&mark[b]), 1u << lane);
                }
            }
            __syncwarp();
            if (lane < cnt) {  // earlier pairs of the step that share a vertex: read off the marks
                const unsigned m = (unsigned)mark[s_lo[lane]] | (unsigned)mark[s_hi[lane]];
                s_share[lane] = m & ((1u << lane) - 1u);
            }
            int incl = len;  // inclusive prefix over lanes
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane < cnt) s_pre[lane + 1] = incl;
            __syncwarp();
            {   // segment table: segment 4j + k (a out, a in, b out, b in of pair j), 32 per pass
                int carry = 0;
                for (int h = 0; h < (4 * CG + 31) / 32; h++) {
                    const int seg = lane + 32 * h, j = seg >> 2, k = seg & 3;
                    const int slen = j < cnt ? s_inf[j][2 * k + 1] : 0;
                    int sincl = slen;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, sincl, o);
                        if (lane >= o) sincl += y;
                    }
                    if (seg < 4 * CG) {
                        s_segpre[seg + 1] = carry + sincl;
                        s_segoff[seg] = j < cnt ? s_inf[j][2 * k] : 0;
                    }
                    carry += __shfl_sync(0xffffffffu, sincl, 31);
                }
                if (lane == 0) s_segpre[0] = 0;
            }
            const unsigned dead = __ballot_sync(0xffffffffu, lane < cnt && (used[s_lo[lane < cnt ? lane : 0]] | used[s_hi[lane < cnt ? lane : 0]]));
            if (lane == 0) {
                s_pre[0] = 0; s_dead = dead;
                s_n = cnt; s_k = k; s_scanned = scanned;
            }
            if (cnt) {
                const int tot = __shfl_sync(0xffffffffu, incl, cnt - 1);
                if (lane == 0) { entries += tot; steps++; }
            }
        } else {   // the other warps clear the step's conditional changes
            for (int q = tid - 32; q < CG * CG; q += blockDim.x - 32) (&s_cc[0][0])[q] = 0;
        }
        __syncthreads();
        const int cnt = s_n;
        if (cnt == 0) break;
        // ---- scan all pairs of the step, entries spread over the CTA; each
        //      thread resolves kMLP entries and issues their loads together ----
        {
            constexpr int kMLP = 4;
            const int all = s_pre[cnt];
            // this CTA's slice of the step's entries
            const int first = (int)((long long)all * ct / nct), tot = (int)((long long)all * (ct + 1) / nct);
            const int nseg = 4 * cnt;
            for (int base = first; base < tot; base += kMLP * blockDim.x) {
                int jj[kMLP], kind[kMLP];
                typename EN::T en[kMLP];
                // this thread's kMLP consecutive entries: one segment search, then
                // step to the next segment where a list ends (coalesced per warp)
                const int e0 = base + kMLP * tid;
                int seg = 0;
                if (e0 < tot) {
                    int lo = 0, hi = nseg;  // s_segpre[lo] <= e0 < s_segpre[hi]
                    while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (s_segpre[mid] <= e0) lo = mid; else hi = mid; }
                    seg = lo;
                }
#pragma unroll
                for (int u = 0; u < kMLP; u++) {
                    const int e = e0 + u;
                    jj[u] = -1;
                    kind[u] = 0;
                    if (e >= tot) continue;
                    while (e >= s_segpre[seg + 1]) seg++;
                    const typename EN::T* src = ((seg & 1) ? g.ent1i : g.ent1o) + s_segoff[seg] + (e - s_segpre[seg]);
                    en[u] = *src;
                    jj[u] = seg >> 2;
                    kind[u] = seg & 3;
                }
                int wv[kMLP][4];
                bool mv[kMLP];
#pragma unroll
                for (int u = 0; u < kMLP; u++) {
                    mv[u] = false;
                    const int j = jj[u];
                    if (j < 0) continue;
                    const int x = EN::id(en[u]);
                    const unsigned im = mark[x] & ((1u << j) - 1u);  // earlier pairs with vertex x
                    if (im) atomicOr(&s_imask[j], im);
                    const int a = s_lo[j], b = s_hi[j];
                    if (x == a || x == b) continue;
                    if (!used[x]) {
                        // x is in earlier pair(s) i of the step: what each one's swap
                        // (x taking its partner's image) would change in this delta
                        for (unsigned rest = im; rest; rest &= rest - 1) {
                            const int i = __ffs(rest) - 1;
                            const int px = p16[s_lo[i] == x ? s_hi[i] : s_lo[i]], qx = p16[x];
                            const int pa = p16[a], pb = p16[b], w = EN::w(en[u]);
                            int c;
                            if (kind[u] == 0 || kind[u] == 2)
                                c = (imin(w, g.w2(pb, px)) - imin(w, g.w2(pa, px))) -
                                    (imin(w, g.w2(pb, qx)) - imin(w, g.w2(pa, qx)));
                            else
                                c = (imin(w, g.w2t(px, pb)) - imin(w, g.w2t(px, pa))) -
                                    (imin(w, g.w2t(qx, pb)) - imin(w, g.w2t(qx, pa)));
                            if (kind[u] >= 2) c = -c;
                            if (c) atomicAdd(&s_cc[j][i], c);
                        }
                        continue;
                    }
                    mv[u] = true;
                    const int pa = p16[a], pb = p16[b], px = p16[x], qx = q16[x];
                    if (kind[u] == 0 || kind[u] == 2) {  // out-edges of the pair's vertex: W2 rows of the images
                        wv[u][0] = g.w2(pb, px); wv[u][1] = g.w2(pa, px); wv[u][2] = g.w2(pb, qx); wv[u][3] = g.w2(pa, qx);
                    } else {                             // in-edges: W2 columns = rows of the transpose
                        wv[u][0] = g.w2t(px, pb); wv[u][1] = g.w2t(px, pa); wv[u][2] = g.w2t(qx, pb); wv[u][3] = g.w2t(qx, pa);
                    }
                }
#pragma unroll
                for (int u = 0; u < kMLP; u++) {
                    if (!mv[u]) continue;
                    const int w = EN::w(en[u]);
                    // a takes p(b) and b takes p(a): the terms of b's edges have the opposite sign
                    int c = (imin(w, wv[u][0]) - imin(w, wv[u][1])) - (imin(w, wv[u][2]) - imin(w, wv[u][3]));
                    if (kind[u] >= 2) c = -c;
                    if (c) atomicAdd(&s_corr[jj[u]], c);
                    atomicAdd(&s_cnt[jj[u]], 1);
                }
            }
        }
        const int my_lo = tid < cnt ? s_lo[tid] : 0, my_hi = tid < cnt ? s_hi[tid] : 0;
        __syncthreads();
        if (nct > 1) {  // exchange the per-pair partial sums of the CTAs' slices
            const int buf = gstep & 1;
            if (tid < cnt) {
                s_cpart[buf][tid][0] = s_corr[tid]; s_cpart[buf][tid][1] = s_cnt[tid];
                s_cpart[buf][tid][2] = (int)s_imask[tid];
            }
            if (tid < cnt * CG) {
                const int j = tid / CG, i = tid - j * CG;
                s_cpart[buf][j][3 + i] = s_cc[j][i];
            }
            __syncthreads();
            if (tid < cnt) { s_corr[tid] = 0; s_cnt[tid] = 0; s_imask[tid] = 0; }
            if (tid < cnt * CG) (&s_cc[0][0])[tid] = 0;
            if (!cluster_step_sync(cbar, (uint32_t)buf, nct, grid.err, grid.stall && gstep == 0)) {
                aborted = true;
                break;
            }
            constexpr int kW = kPart / 4;   // 16-byte words per pair
            for (int t = tid; t < nct * cnt * kW; t += blockDim.x) {
                // (c, j, w): word w of CTA c's partials of pair j (integer sums: any order)
                const int c = t / (cnt * kW), r = t - c * (cnt * kW);
                const int j = r / kW, w = r - j * kW;
                const uint32_t q = cluster_map((uint32_t)__cvta_generic_to_shared(&s_cpart[buf][j][4 * w]), (uint32_t)c);
                int v[4];
                asm volatile("ld.shared::cluster.v4.u32 {%0, %1, %2, %3}, [%4];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "r"(q) : "memory");
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int k = 4 * w + u;
                    if (!v[u] || k >= 3 + CG) continue;
                    if (k == 0) atomicAdd(&s_corr[j], v[u]);
                    else if (k == 1) atomicOr(&s_cnt[j], v[u]);
                    else if (k == 2) atomicOr(&s_imask[j], (unsigned)v[u]);
                    else atomicAdd(&s_cc[j][k - 3], v[u]);
                }
            }
            __syncthreads();
        }
        gstep++;
        // ---- clear the step's marks; decide in order in warp 0: lane j holds pair
        //      j's fields, every lane replays the same bitmask logic over the
        //      shuffled fields, then the lanes apply their own outcomes ----
        if (tid < cnt) { mark[my_lo] = 0; mark[my_hi] = 0; }
        if (wid == 0) {
            const bool in = lane < cnt;
            const unsigned share = in ? s_share[lane] : 0u, adj = in ? s_imask[lane] : 0u;
            const int moved = in ? s_cnt[lane] : 0, d0 = in ? s_d0[lane] : 0;
            int corr = in ? s_corr[lane] : 0;   // grows by cc[lane][i] when earlier pair i commits
            const int a = in ? s_lo[lane] : 0, b = in ? s_hi[lane] : 0;
            const unsigned dead = s_dead;
            unsigned cm = 0;
#pragma unroll
            for (int j = 0; j < CG; j++) {
                const unsigned sh_j = __shfl_sync(0xffffffffu, share, j);
                const unsigned ad_j = __shfl_sync(0xffffffffu, adj, j);
                const int mv_j = __shfl_sync(0xffffffffu, moved, j);
                const int co_j = __shfl_sync(0xffffffffu, corr, j);
                const int d0_j = __shfl_sync(0xffffffffu, d0, j);
                if (j >= cnt) continue;
                if (((dead >> j) & 1u) || (sh_j & cm)) continue;   // a vertex already moved: skip
                int d = d0_j;
                bool ok = true;
                if (mv_j > 0 || (ad_j & cm)) {                   // next to a moved vertex: re-verify
                    if (max_verify >= 0 && verified >= max_verify) ok = false;
                    else { verified++; d += co_j; }
                }
                if (ok && d > 0) {
                    cm |= 1u << j;
                    total += d;
                    committed++;
                    if (lane > j && lane < cnt) corr += s_cc[lane][j];
                }
            }
            __syncwarp();
            if ((cm >> lane) & 1u) {  // committed pairs share no vertex: apply in parallel
                const int fa = p16[a], fb = p16[b];
                q16[a] = (uint16_t)fa; q16[b] = (uint16_t)fb;
                p16[a] = (uint16_t)fb; p16[b] = (uint16_t)fa;
                if (ct == 0) {
                    if (fb < n) g.pinv[fb] = a;
                    if (fa < n) g.pinv[fa] = b;
                }
                used[a] = 1; used[b] = 1;
            }
            if (lane == 0) s_n = 0;
        }
        __syncthreads();
    }
    if (nct > 1 && !aborted) cluster_step_sync(cbar, (uint32_t)(gstep & 1), nct, grid.err);
    if (ct != 0) return;
    for (int i = tid; i < n; i += blockDim.x) g.p[i] = p16[i];
    if (tid == 0) {
        st->total_delta = total;
        st->scanned = s_scanned;
        st->verified = verified;
        st->committed = committed;
        st->steps = steps;
        st->entries = entries;
        st->carried = 0;   // every pair is decided in the step that scans it
    }
}

// Pulls [p, p + bytes) into L2 (one prefetch per 128-byte line).  The set
// commit reads G1 list entries of scattered vertices from a single CTA; the
// profit matrix traffic before it has evicted those lists, so without this
// every first touch of a list goes to HBM.
static __global__ void k_prefetch_l2(const char* __restrict__ p, size_t bytes) {
    const size_t lines = (bytes + 127) / 128;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < lines; i += (size_t)gridDim.x * blockDim.x)
        asm volatile("prefetch.global.L2 [%0];" :: "l"(p + i * 128));
}

// List extents of each sorted candidate for the set commit, two int4 per
// candidate: (out-offset, out-length, in-offset, in-length) of its lower and of
// its higher vertex; zeros for the "no candidate" key ~0.
template <bool W16>
__global__ void k_cand_info(DevView<W16> g, const unsigned long long* __restrict__ keys, int lim,
                            int4* __restrict__ info) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lim) return;
    const unsigned long long key = keys[i];
    int4 x = make_int4(0, 0, 0, 0), y = x;
    if (key != ~0ull) {
        const int lo = (int)((key >> 16) & 0xffffu), hi = (int)(key & 0xffffu);
        x.x = g.off1o[lo]; x.y = g.off1o[lo + 1] - x.x; x.z = g.off1i[lo]; x.w = g.off1i[lo + 1] - x.z;
        y.x = g.off1o[hi]; y.y = g.off1o[hi + 1] - y.x; y.z = g.off1i[hi]; y.w = g.off1i[hi + 1] - y.z;
    }
    info[2 * i] = x;
    info[2 * i + 1] = y;
}

constexpr int kCommitMaxCtas = 8;      // a portable cluster
constexpr int kCommitDefaultCtas = 8;
// The set commit's error word (one int; bit 1: a cluster wait ran out).
__host__ __device__ inline size_t commit_grid_ints() { return 4; }

// Launches the set commit on `ctas` CTAs forming one thread-block cluster (a
// plain launch for one); `buf` holds commit_grid_ints() ints: the error word,
// reset here.  Returns the launch status.
template <bool W16>
__host__ inline cudaError_t launch_commit_group(const DevView<W16>& g, const unsigned long long* keys, int lim,
                                               int max_verify, CommitStats* st, const int4* cinfo, int ctas,
                                               int* buf, size_t smem, cudaStream_t stream, int stall = 0);

// Shared memory bytes of commit_group for n vertices (used flags, matching,
// pre-move images, step marks of mark_bytes each).
__host__ __device__ inline size_t commit_group_smem(int n, int mark_bytes = 2) {
    return (size_t)((n + 15) & ~15) + (4 + mark_bytes) * (size_t)((n + 8) & ~7);
}

template <bool W16, int CG = kCG>
__global__ void __launch_bounds__(1024)
k_commit_group(DevView<W16> g, const unsigned long long* __restrict__ keys, int lim, int max_verify,
               CommitStats* __restrict__ st, const int4* __restrict__ cinfo, CommitGrid grid) {
    extern __shared__ unsigned char smem[];
    commit_group<W16, CG>(g, keys, lim, max_verify, st, smem, cinfo, grid);
}

template <bool W16>
__host__ inline cudaError_t launch_commit_group(const DevView<W16>& g, const unsigned long long* keys, int lim,
                                               int max_verify, CommitStats* st, const int4* cinfo, int ctas,
                                               int* buf, size_t smem, cudaStream_t stream, int stall) {
    cudaError_t e = cudaFuncSetAttribute(k_commit_group<W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    CommitGrid grid{1, buf, stall};
    if (ctas <= 1) {
        k_commit_group<W16><<<1, 1024, smem, stream>>>(g, keys, lim, max_verify, st, cinfo, grid);
        return cudaGetLastError();
    }
    // a cluster decides 32 pairs per step when 32-bit marks fit (n up to about
    // 23,000), else 16
    bool wide = false;
    const size_t wsmem = commit_group_smem(g.n, 4);
    if (cudaFuncSetAttribute(k_commit_group<W16, kCGWide>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsmem) ==
        cudaSuccess) {
        int per_sm = 0;
        wide = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_commit_group<W16, kCGWide>, 1024, wsmem) ==
                   cudaSuccess && per_sm >= 1;
    }
    cudaGetLastError();   // a refused attribute is not an error of this launch
    grid.nct = ctas;
    if ((e = cudaMemsetAsync(grid.err, 0, sizeof(int), stream)) != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = wide ? wsmem : smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (wide) return cudaLaunchKernelEx(&cfg, k_commit_group<W16, kCGWide>, g, keys, lim, max_verify, st, cinfo, grid);
    return cudaLaunchKernelEx(&cfg, k_commit_group<W16>, g, keys, lim, max_verify, st, cinfo, grid);
}

}  // namespace bm
