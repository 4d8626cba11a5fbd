// GETRF panel, pivot composition and row-permutation kernels (FP32).
//
// getf2_coop replaces rocsolver_sgetrf's unblocked leaf on the tall panel
// (src/getrf/getrf_pivot_internal.h:17-39): one cooperative launch factors an
// m x w (w <= 128) column block with partial pivoting.  Each CTA keeps a
// contiguous slice of rows of the block resident in shared memory; per column
// the CTAs publish their local |max| candidate (value, row and the full
// candidate row) and the owner of the diagonal row publishes that row, then
// exchange them through global memory (see the protocol note below), after
// which every CTA picks the same global winner (largest |a|, lowest row on
// ties -- LAPACK ISAMAX), swaps, scales by the reciprocal pivot (division
// when |pivot| < FLT_MIN, as xGETF2) and applies the rank-1 update to its own
// rows -- the next column first, so that its candidate is published before
// the rest of the update runs.
//
// compose_swaps + apply_moves replace apply_panel_pivots_kernel
// (src/getrf/getrf_pivot_kernels.hip:14-45) and the host-side permutation
// batching (src/getrf/getrf_batched_pivot_internal.h:59-223): a LAPACK swap
// sequence is composed on the GPU into a list of (source, target) row moves,
// then applied to column tiles with a gather into shared memory followed by a
// scatter -- no host round trip.
#include <cfloat>
#include <climits>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int kCoopThreads = 256;
constexpr int kCoopMaxW = 128;
constexpr int kCoopMaxGrid = 256;
// Per-(parity, CTA) exchange slot, in 64-bit words:
// [header, pad | candidate row (kCoopMaxW) | diagonal row (kCoopMaxW)]
constexpr int kSlotWords = 2 + 2 * kCoopMaxW;

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Candidate (v, i) beats (bv, bi): a real row beats none, then larger |a|,
// then the lower row (LAPACK ISAMAX returns the first maximum).
__device__ __forceinline__ bool better(float v, int i, float bv, int bi)
{
    if (i == INT_MAX) return false;
    if (bi == INT_MAX) return true;
    return v > bv || (v == bv && i < bi);
}

// Copy an nr x w column block between global memory and the shared tile
// (leading dimension ldt), eight independent loads in flight per thread.
template <bool TO_SMEM>
__device__ __forceinline__ void coop_move(float* A, long long lda, float* tile, int ldt, int nr,
                                          int w)
{
    const int total = nr * w;
    int e = threadIdx.x;
    for (; e + 7 * kCoopThreads < total; e += 8 * kCoopThreads) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kCoopThreads, c = q / nr, r = q - c * nr;
            v[u] = TO_SMEM ? A[(long long)c * lda + r] : tile[c * ldt + r];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kCoopThreads, c = q / nr, r = q - c * nr;
            if (TO_SMEM) tile[c * ldt + r] = v[u];
            else A[(long long)c * lda + r] = v[u];
        }
    }
    for (; e < total; e += kCoopThreads) {
        const int c = e / nr, r = e - c * nr;
        if (TO_SMEM) tile[c * ldt + r] = A[(long long)c * lda + r];
        else A[(long long)c * lda + r] = tile[c * ldt + r];
    }
}

constexpr unsigned kNoRow = 0xffffu;  // "no candidate" in the header

// Exchange protocol (no grid barrier, no fences).  Slot (parity, CTA) holds
// 64-bit words, each written and read whole (single-copy atomic):
//   header  [ |a| bits : 32 | column + 1 : 16 | local row : 16 ]
//   rows    [ tag : 32 | value bits : 32 ] for the CTA's candidate row and,
//           from the CTA owning it, the diagonal row; tag = epoch << 8 |
//           column + 1, epoch = launch counter.
// Column j uses parity j & 1.  Every CTA polls all G headers (thread q
// watches CTA q, bounded) and then reads the winner's and the diagonal rows,
// re-reading any word whose tag is not yet this column's: each word proves
// its own freshness, so a writer needs no release fence between its rows and
// its header, and one L2 trip delivers the flag with the candidate.  A CTA
// only rewrites a parity after every CTA has published the following column,
// i.e. after all of them finished reading it, so two parities suffice.  The
// last CTA to finish zeroes every header (column 0 never matches) and
// advances the epoch, so no launch accepts an earlier launch's words.
//
// Look-ahead inside the column loop: after the pivot of column j is applied,
// each CTA updates only column j + 1 of its rows, publishes its column-(j+1)
// candidate and then runs the rest of the rank-1 update while the exchange
// is in flight.  The published rows therefore still lack step j's update in
// columns > j + 1; the receivers finish them with the row's own multiplier
// (its column-j entry) and the step-j pivot row -- the same fmaf the owner
// applies to its copy, so every CTA holds bit-identical rows.
__global__ void __launch_bounds__(kCoopThreads)
getf2_coop_kernel(int m, int w, float* A, long long lda, int rpc, int* ipiv, int ipiv_add,
                  int* info, int info_base, unsigned long long* scr, unsigned* epoch_ptr,
                  unsigned* done_ptr, int* err, int pivot)
{
    extern __shared__ float tile[];  // tile[c * rpc + r]
    __shared__ float prow_s[2][kCoopMaxW];  // pivot rows of the last two columns
    __shared__ float red_v[kCoopThreads / 32];
    __shared__ int red_i[kCoopThreads / 32];
    __shared__ float cv[kCoopMaxGrid];
    __shared__ int ci[kCoopMaxGrid];
    __shared__ int s_abort, s_last;

    const int G = gridDim.x;
    const int cta = blockIdx.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int r0 = cta * rpc;
    const int nr = max(0, min(m, r0 + rpc) - r0);
    const int steps = min(m, w);
    const unsigned epoch = *reinterpret_cast<volatile unsigned*>(epoch_ptr);
    const unsigned spin = spin_limit_of(err);
    auto slot_of = [&](int par, int q) {
        return scr + ((long long)par * kCoopMaxGrid + q) * kSlotWords;
    };
    auto row_tag = [&](int col) { return (epoch << 8) | (unsigned)(col + 1); };

    coop_move<true>(A + r0, lda, tile, rpc, nr, w);
    if (tid == 0) s_abort = 0;
    __syncthreads();

    // Block-wide candidate of column `col` over owned rows >= col, from the
    // values now in the tile; every thread returns the same local row (or -1).
    auto block_candidate = [&](int col, float& val) -> int {
        float bv = -1.f;
        int bi = INT_MAX;
        for (int r = tid; r < nr; r += kCoopThreads) {
            if (r0 + r >= col) {
                const float v = fabsf(tile[col * rpc + r]);
                if (bi == INT_MAX || v > bv) { bv = v; bi = r0 + r; }
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float ov = __shfl_down_sync(0xffffffffu, bv, off);
            const int oi = __shfl_down_sync(0xffffffffu, bi, off);
            if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
        }
        if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
        __syncthreads();
        bv = red_v[0];
        bi = red_i[0];
#pragma unroll
        for (int q = 1; q < kCoopThreads / 32; ++q)
            if (better(red_v[q], red_i[q], bv, bi)) { bv = red_v[q]; bi = red_i[q]; }
        val = bv;
        return bi == INT_MAX ? -1 : bi - r0;
    };

    // Publish column `col`: candidate row (local index lr, or -1), the
    // diagonal row if owned, and the header (no ordering needed among them).
    auto publish = [&](int col, int lr, float val) {
        unsigned long long* slot = slot_of(col & 1, cta);
        const unsigned long long t = (unsigned long long)row_tag(col) << 32;
        const bool own_diag = col >= r0 && col < r0 + nr;
        if (tid < w) {
            if (lr >= 0) st_relaxed_u64(slot + 2 + tid, t | __float_as_uint(tile[tid * rpc + lr]));
            if (own_diag)
                st_relaxed_u64(slot + 2 + kCoopMaxW + tid,
                               t | __float_as_uint(tile[tid * rpc + (col - r0)]));
        }
        if (tid == 0) {
            const unsigned lo = ((unsigned)(col + 1) << 16) | (lr >= 0 ? (unsigned)lr : kNoRow);
            const unsigned hi = lr >= 0 ? __float_as_uint(val) : __float_as_uint(-1.f);
            st_relaxed_u64(slot, ((unsigned long long)hi << 32) | lo);
        }
        __syncthreads();  // the rows were read before the rank-1 update rewrites them
    };

    if (steps > 0) {  // column 0 candidates, nothing to finish on the receiving side
        float v = -1.f;
        int lr = -1;
        if (pivot) lr = block_candidate(0, v);
        publish(0, lr, v);
    }

    for (int j = 0; j < steps; ++j) {
        const int par = j & 1;
        const unsigned tag = (unsigned)j + 1u;

        // 1. every candidate header of column j (thread q watches CTA q), bounded
        for (int q = tid; q < G; q += kCoopThreads) {
            const unsigned long long* wq = slot_of(par, q);
            unsigned polls = 0;
            unsigned long long wv;
            while (((unsigned)((wv = ld_relaxed_u64(wq)) >> 16) & 0xffffu) != tag) {
                if (++polls > spin) {
                    atomicCAS(err, 0, kErrTimeout);
                    s_abort = 1;
                    break;
                }
                if (polls > 256) __nanosleep(32);
            }
            const unsigned lr = (unsigned)wv & 0xffffu;
            cv[q] = __uint_as_float((unsigned)(wv >> 32));
            ci[q] = lr == kNoRow ? INT_MAX : q * rpc + (int)lr;
        }
        __syncthreads();
        if (s_abort) break;

        // 2. the winner (each of the first warps reduces redundantly), its
        // row and the diagonal row, finished with step j-1's update; swap.
        const int owner = j / rpc;
        float* prow = prow_s[par];
        const float* prev = prow_s[par ^ 1];
        if (tid < ((w + 31) & ~31)) {
            int gi = j, gc = owner;
            if (pivot) {
                float gv = -1.f;
                gi = INT_MAX;
                for (int q = lane; q < G; q += 32)
                    if (better(cv[q], ci[q], gv, gi)) { gv = cv[q]; gi = ci[q]; gc = q; }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const float ov = __shfl_xor_sync(0xffffffffu, gv, off);
                    const int oi = __shfl_xor_sync(0xffffffffu, gi, off);
                    const int oc = __shfl_xor_sync(0xffffffffu, gc, off);
                    if (better(ov, oi, gv, gi)) { gv = ov; gi = oi; gc = oc; }
                }
                if (gi == INT_MAX) { gi = j; gc = owner; }  // unreachable: row j always competes
            }
            if (tid < w) {
                // without pivoting the pivot row is the diagonal row
                const unsigned long long* sw =
                    pivot ? slot_of(par, gc) + 2 : slot_of(par, owner) + 2 + kCoopMaxW;
                const unsigned long long* so = slot_of(par, owner) + 2 + kCoopMaxW;
                const unsigned want = row_tag(j);
                const bool fin = j > 0 && tid > j;
                unsigned long long wp = ld_relaxed_u64(sw + tid), wo = ld_relaxed_u64(so + tid);
                unsigned long long wl = fin ? ld_relaxed_u64(sw + (j - 1)) : 0ull;
                unsigned long long wm = fin ? ld_relaxed_u64(so + (j - 1)) : 0ull;
                unsigned polls = 0;
                while ((unsigned)(wp >> 32) != want || (unsigned)(wo >> 32) != want ||
                       (fin && ((unsigned)(wl >> 32) != want || (unsigned)(wm >> 32) != want))) {
                    if (++polls > spin) {
                        atomicCAS(err, 0, kErrTimeout);
                        s_abort = 1;
                        break;
                    }
                    wp = ld_relaxed_u64(sw + tid);
                    wo = ld_relaxed_u64(so + tid);
                    if (fin) {
                        wl = ld_relaxed_u64(sw + (j - 1));
                        wm = ld_relaxed_u64(so + (j - 1));
                    }
                }
                float pv = __uint_as_float((unsigned)wp), ov = __uint_as_float((unsigned)wo);
                if (fin) {
                    pv = fmaf(-__uint_as_float((unsigned)wl), prev[tid], pv);
                    ov = fmaf(-__uint_as_float((unsigned)wm), prev[tid], ov);
                }
                prow[tid] = pv;
                if (gi != j) {
                    if (j >= r0 && j < r0 + nr) tile[tid * rpc + (j - r0)] = pv;
                    if (gi >= r0 && gi < r0 + nr) tile[tid * rpc + (gi - r0)] = ov;
                }
            }
            if (tid == 0 && pivot && cta == 0) ipiv[j] = gi + 1 + ipiv_add;
        }
        __syncthreads();
        if (s_abort) break;

        // 3. scale column j, update column j+1 and find its candidate
        const float piv = prow[j];
        const bool nz = piv != 0.f;
        const bool recip = fabsf(piv) >= FLT_MIN;
        const float rcp = 1.0f / piv;
        if (!nz && cta == 0 && tid == 0 && info) atomicCAS(info, 0, info_base + j + 1);
        const bool next = j + 1 < w;
        const float pn = next ? prow[j + 1] : 0.f;
        for (int r = tid; r < nr; r += kCoopThreads) {
            if (r0 + r > j) {
                float l = tile[j * rpc + r];
                if (nz) {
                    l = recip ? l * rcp : l / piv;
                    tile[j * rpc + r] = l;
                }
                if (next) tile[(j + 1) * rpc + r] = fmaf(-l, pn, tile[(j + 1) * rpc + r]);
            }
        }
        if (j + 1 < steps) {
            float v = -1.f;
            int lr = -1;
            if (pivot) lr = block_candidate(j + 1, v);  // its barrier orders the updates above
            else __syncthreads();
            publish(j + 1, lr, v);
        }

        // 4. the rest of step j's rank-1 update, overlapping the exchange
        for (int r = tid; r < nr; r += kCoopThreads) {
            if (r0 + r > j) {
                const float l = tile[j * rpc + r];
                int c = j + 2;
                for (; c + 3 < w; c += 4) {
                    const float t0 = tile[c * rpc + r], t1 = tile[(c + 1) * rpc + r];
                    const float t2 = tile[(c + 2) * rpc + r], t3 = tile[(c + 3) * rpc + r];
                    tile[c * rpc + r] = fmaf(-l, prow[c], t0);
                    tile[(c + 1) * rpc + r] = fmaf(-l, prow[c + 1], t1);
                    tile[(c + 2) * rpc + r] = fmaf(-l, prow[c + 2], t2);
                    tile[(c + 3) * rpc + r] = fmaf(-l, prow[c + 3], t3);
                }
                for (; c < w; ++c) tile[c * rpc + r] = fmaf(-l, prow[c], tile[c * rpc + r]);
            }
        }
    }
    __syncthreads();

    coop_move<false>(A + r0, lda, tile, rpc, nr, w);

    // The last CTA to finish clears every header of this launch and moves
    // the epoch on.
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(done_ptr, 1u) + 1u == (unsigned)G;
    }
    __syncthreads();
    if (s_last) {
        for (int q = tid; q < 2 * G; q += kCoopThreads) *slot_of(q / G, q % G) = 0ull;
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicExch(done_ptr, 0u);
            atomicAdd(epoch_ptr, 1u);
        }
    }
}

// ------------------------------------------------------------ compose swaps
constexpr int kComposeThreads = 1024;
constexpr int kComposeMaxK = 4096;  // swaps composed by the sorted-group kernels

__host__ __device__ constexpr int pow2_at_least(int v)
{
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Block-wide ordered compaction: items q = 0 .. total-1 in order, item q
// kept when pick(q, &s, &t) is true; kept items are written to src/tgt at
// base + (rank among kept items).  Returns the new base (uniform).
template <class Pick>
__device__ int emit_ordered(int total, int base, int* src, int* tgt, int* warp_tot, int* s_chunk,
                            Pick pick)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int q0 = 0; q0 < total; q0 += kComposeThreads) {
        const int q = q0 + tid;
        int s = 0, t = 0;
        const bool moved = q < total && pick(q, &s, &t);
        const unsigned ball = __ballot_sync(0xffffffffu, moved);
        const int within = __popc(ball & ((1u << lane) - 1u));
        if (lane == 0) warp_tot[warp] = __popc(ball);
        __syncthreads();
        if (tid == 0) {
            int run = 0;
            for (int wv = 0; wv < kComposeThreads / 32; ++wv) {
                const int c = warp_tot[wv];
                warp_tot[wv] = run;
                run += c;
            }
            *s_chunk = run;
        }
        __syncthreads();
        if (moved) {
            src[base + warp_tot[warp] + within] = s;
            tgt[base + warp_tot[warp] + within] = t;
        }
        base += *s_chunk;
        __syncthreads();
    }
    return base;
}

// Composition of a LAPACK swap sequence without replaying it.  Step t
// (t = 0 .. kk-1) exchanges the contents of position x_t = base + t with
// position bt[t] >= x_t.  Position x_t is never touched after step t, and a
// position p >= x_t is touched before step t only by the steps j < t with
// bt[j] = p.  So, with the (bt, t) pairs sorted:
//   prev(t) = the last j < t with bt[j] = bt[t]      (same-target group)
//   g(u)    = the last j < u with bt[j] = x_u        (who filled x_u before step u)
//   V(u)    = content of x_u just before step u = start(x_{root(u)}), root(u)
//             the end of the chain u -> g(u) -> g(g(u)) ... (pointer jumping)
// and the contents after the whole sequence are
//   position x_t:                 prev(t) >= 0 ? V(prev(t)) : start(bt[t])
//   target p >= base + kk (last t of its group): V(t).
// Results: nv[t] (content of x_t), keys[s] the sorted pairs, root[u] the chain
// ends; aux[t] holds prev(t).  start() must stay valid until the caller writes
// the new contents.
template <class Start>
__device__ void compose_sorted(const int* bt, int kk, int base, int P, unsigned long long* keys,
                               int* aux, int* root, int* nv, Start start)
{
    const int tid = threadIdx.x;
    for (int s = tid; s < P; s += kComposeThreads)
        keys[s] = s < kk ? ((unsigned long long)(unsigned)bt[s] << 32) | (unsigned)s : ~0ull;
    for (int u = tid; u < kk; u += kComposeThreads) root[u] = -1;
    __syncthreads();
    // bitonic sort, ascending (b, t)
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = tid; i < P / 2; i += kComposeThreads) {
                const int lo = 2 * i - (i & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const unsigned long long a = keys[lo], b = keys[hi];
                if ((a > b) == up) {
                    keys[lo] = b;
                    keys[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    for (int s = tid; s < kk; s += kComposeThreads) {
        const unsigned long long key = keys[s];
        const int b = (int)(key >> 32), t = (int)(key & 0xffffffffu);
        const bool has_prev = s > 0 && (int)(keys[s - 1] >> 32) == b;
        aux[t] = has_prev ? (int)(keys[s - 1] & 0xffffffffu) : -1;
        const int u = b - base;  // b is the swap-side position of step u
        if (u < kk && t < u) {
            const bool next_in = s + 1 < kk && (int)(keys[s + 1] >> 32) == b;
            if (!next_in || (int)(keys[s + 1] & 0xffffffffu) == u) root[u] = t;
        }
    }
    __syncthreads();
    for (int u = tid; u < kk; u += kComposeThreads)
        if (root[u] < 0) root[u] = u;
    __syncthreads();
    // Pointer jumping: every root[] value is an ancestor, so reading an entry
    // another thread is updating in the same round is harmless; a round in
    // which nothing changes has read only settled values.
    for (;;) {
        int changed = 0;
        for (int u = tid; u < kk; u += kComposeThreads) {
            const int r = root[u], rr = root[r];
            if (rr != r) {
                root[u] = rr;
                changed = 1;
            }
        }
        if (!__syncthreads_or(changed)) break;
    }
    for (int t = tid; t < kk; t += kComposeThreads) {
        const int p = aux[t];
        nv[t] = p >= 0 ? start(base + root[p]) : start(bt[t]);
    }
    __syncthreads();
}

// Shared-memory layout of the sorted-group kernels (after `lead` ints):
// keys[P] (8-byte aligned), then bt, aux, root, nv (kk ints each).
__host__ __device__ inline size_t compose_sorted_bytes(int lead, int kk)
{
    const size_t head = ((size_t)lead * sizeof(int) + 15) / 16 * 16;
    return head + (size_t)pow2_at_least(kk < 1 ? 1 : kk) * 8 + 4 * (size_t)kk * sizeof(int);
}

// Swaps ipiv[0..k) (rows local after subtracting 1 + ipiv_minus) composed
// into the row moves of A(0:m, :): rows [0, k) in order, then the distinct
// pivot rows >= k in increasing order.  Touches O(k) rows only.
__global__ void __launch_bounds__(kComposeThreads)
compose_swaps_kernel(const int* __restrict__ ipiv, int k, int ipiv_minus, int m, int* src,
                     int* tgt, int* count, int* info, int* err)
{
    extern __shared__ __align__(16) unsigned char craw[];
    __shared__ int warp_tot[kComposeThreads / 32];
    __shared__ int s_bad, s_chunk;
    const int P = pow2_at_least(k);
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(craw);
    int* bt = reinterpret_cast<int*>(keys + P);
    int* aux = bt + k;
    int* root = aux + k;
    int* nv = root + k;
    const int tid = threadIdx.x;
    if (tid == 0) s_bad = 0;
    __syncthreads();
    for (int i = tid; i < k; i += kComposeThreads) {
        const int b = ipiv[i] - 1 - ipiv_minus;
        if (b < i || b >= m) s_bad = 1;
        bt[i] = b;
    }
    __syncthreads();
    if (s_bad) {
        if (tid == 0) {
            *count = 0;
            if (info) atomicExch(info, -1);
            atomicCAS(err, 0, kErrBadPivot);
        }
        return;
    }
    compose_sorted(bt, k, 0, P, keys, aux, root, nv, [](int x) { return x; });
    int base = emit_ordered(k, 0, src, tgt, warp_tot, &s_chunk, [&](int q, int* s, int* t) {
        *s = nv[q];
        *t = q;
        return nv[q] != q;
    });
    base = emit_ordered(k, base, src, tgt, warp_tot, &s_chunk, [&](int q, int* s, int* t) {
        const unsigned long long key = keys[q];
        const int b = (int)(key >> 32);
        if (b < k || (q + 1 < k && (int)(keys[q + 1] >> 32) == b)) return false;
        *s = root[(int)(key & 0xffffffffu)];
        *t = b;
        return *s != b;
    });
    if (tid == 0) *count = base;
}

// The same composition by replaying the swaps in one thread, for sequences
// longer than kComposeMaxK: perm[m] (shared memory, or global scratch when
// it does not fit), then the same move order.
__global__ void __launch_bounds__(kComposeThreads)
compose_swaps_serial_kernel(const int* __restrict__ ipiv, int k, int ipiv_minus, int m,
                            int* src, int* tgt, int* count, int* gperm, int use_smem, int* info,
                            int* err)
{
    extern __shared__ int sperm[];
    __shared__ int warp_tot[kComposeThreads / 32];
    __shared__ int s_bad, s_chunk;
    int* perm = use_smem ? sperm : gperm;
    const int tid = threadIdx.x;
    if (tid == 0) s_bad = 0;
    __syncthreads();
    for (int q = tid; q < m; q += kComposeThreads) perm[q] = q;
    for (int i = tid; i < k; i += kComposeThreads) {
        const int b = ipiv[i] - 1 - ipiv_minus;
        if (b < i || b >= m) s_bad = 1;
    }
    __syncthreads();
    if (s_bad) {
        if (tid == 0) {
            *count = 0;
            if (info) atomicExch(info, -1);
            atomicCAS(err, 0, kErrBadPivot);
        }
        return;
    }
    if (tid == 0) {
        for (int i = 0; i < k; ++i) {
            const int b = ipiv[i] - 1 - ipiv_minus;
            const int t = perm[i];
            perm[i] = perm[b];
            perm[b] = t;
        }
    }
    __syncthreads();
    int base = emit_ordered(k, 0, src, tgt, warp_tot, &s_chunk, [&](int q, int* s, int* t) {
        *s = perm[q];
        *t = q;
        return perm[q] != q;
    });
    // pivot rows >= k: each distinct row once, in increasing row order
    base = emit_ordered(m - k, base, src, tgt, warp_tot, &s_chunk, [&](int q, int* s, int* t) {
        *s = perm[k + q];
        *t = k + q;
        return perm[k + q] != k + q;
    });
    if (tid == 0) *count = base;
}

// Running composition for the GETRF look-ahead: the block's permutation pos[m]
// (position -> source row, kept in global memory between launches) is staged
// in shared memory, the new swaps ipiv[k0..k1) are composed on top of it by
// the sorted-group method, and every displaced row of the block becomes a
// move, in increasing target order.
__global__ void __launch_bounds__(kComposeThreads)
compose_running_kernel(const int* __restrict__ ipiv, int k0, int k1, int ipiv_minus, int m,
                       int* pos, int init, int* src, int* tgt, int* count, int* info, int* err)
{
    extern __shared__ __align__(16) unsigned char craw[];
    __shared__ int warp_tot[kComposeThreads / 32];
    __shared__ int s_bad, s_chunk;
    const int kk = k1 - k0;
    const int P = pow2_at_least(kk < 1 ? 1 : kk);
    int* sp = reinterpret_cast<int*>(craw);
    unsigned long long* keys =
        reinterpret_cast<unsigned long long*>(craw + ((size_t)m * sizeof(int) + 15) / 16 * 16);
    int* bt = reinterpret_cast<int*>(keys + P);
    int* aux = bt + kk;
    int* root = aux + kk;
    int* nv = root + kk;
    const int tid = threadIdx.x;
    if (tid == 0) s_bad = 0;
    __syncthreads();
    for (int q = tid; q < m; q += kComposeThreads) sp[q] = init ? q : pos[q];
    for (int t = tid; t < kk; t += kComposeThreads) {
        const int b = ipiv[k0 + t] - 1 - ipiv_minus;
        if (b < k0 + t || b >= m) s_bad = 1;
        bt[t] = b;
    }
    __syncthreads();
    if (s_bad) {
        if (tid == 0) {
            *count = 0;
            if (info) atomicExch(info, -1);
            atomicCAS(err, 0, kErrBadPivot);
        }
        return;
    }
    if (kk > 0) {
        compose_sorted(bt, kk, k0, P, keys, aux, root, nv, [&](int x) { return sp[x]; });
        // final contents of the targets beyond the swapped rows (aux reused)
        for (int s = tid; s < kk; s += kComposeThreads) {
            const unsigned long long key = keys[s];
            const int b = (int)(key >> 32);
            const bool last = !(s + 1 < kk && (int)(keys[s + 1] >> 32) == b);
            aux[s] = (last && b >= k1) ? sp[k0 + root[(int)(key & 0xffffffffu)]] : -1;
        }
        __syncthreads();
        for (int t = tid; t < kk; t += kComposeThreads) {
            sp[k0 + t] = nv[t];
            if (aux[t] >= 0) sp[(int)(keys[t] >> 32)] = aux[t];
        }
        __syncthreads();
    }
    for (int q = tid; q < m; q += kComposeThreads) pos[q] = sp[q];
    const int base = emit_ordered(m, 0, src, tgt, warp_tot, &s_chunk, [&](int q, int* s, int* t) {
        *s = sp[q];
        *t = q;
        return sp[q] != q;
    });
    if (tid == 0) *count = base;
}

// ------------------------------------------------------------ apply moves
constexpr int kApplyThreads = 256;

// Columns [blockIdx.x*cpc, +cpc): gather every source row into shared memory,
// then scatter to the targets.  Sources and targets are the same row set, so
// reading everything before writing anything is race-free per column.
__global__ void __launch_bounds__(kApplyThreads)
apply_moves_smem_kernel(float* A, long long lda, int ncols, const int* __restrict__ src,
                        const int* __restrict__ tgt, const int* __restrict__ count, int cpc,
                        int cap)
{
    extern __shared__ float buf[];  // cpc * cap values, then cap sources, cap targets
    int* s_src = reinterpret_cast<int*>(buf + (size_t)cpc * cap);
    int* s_tgt = s_src + cap;
    const int cnt = min(*count, cap);
    if (cnt <= 0) return;
    const int c0 = blockIdx.x * cpc;
    const int nc = min(cpc, ncols - c0);
    for (int i = threadIdx.x; i < cnt; i += kApplyThreads) {
        s_src[i] = src[i];
        s_tgt[i] = tgt[i];
    }
    __syncthreads();
    // Flattened (column, move) space, eight independent loads in flight.
    const int total = nc * cnt;
    const float* base = A + (long long)c0 * lda;
    int e = threadIdx.x;
    for (; e + 7 * kApplyThreads < total; e += 8 * kApplyThreads) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kApplyThreads, cc = q / cnt, i = q - cc * cnt;
            v[u] = base[(long long)cc * lda + s_src[i]];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kApplyThreads, cc = q / cnt, i = q - cc * cnt;
            buf[cc * cap + i] = v[u];
        }
    }
    for (; e < total; e += kApplyThreads) {
        const int cc = e / cnt, i = e - cc * cnt;
        buf[cc * cap + i] = base[(long long)cc * lda + s_src[i]];
    }
    __syncthreads();
    float* wbase = A + (long long)c0 * lda;
    for (int q = threadIdx.x; q < total; q += kApplyThreads) {
        const int cc = q / cnt, i = q - cc * cnt;
        wbase[(long long)cc * lda + s_tgt[i]] = buf[cc * cap + i];
    }
}

__global__ void gather_rows_kernel(const float* A, long long lda, int ncols,
                                   const int* __restrict__ src, const int* __restrict__ count,
                                   int cap, float* temp)
{
    const int cnt = min(*count, cap);
    const long long total = (long long)cnt * ncols;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % cnt);
        const long long c = idx / cnt;
        temp[c * cap + i] = A[c * lda + src[i]];
    }
}

__global__ void scatter_rows_kernel(float* A, long long lda, int ncols,
                                    const int* __restrict__ tgt, const int* __restrict__ count,
                                    int cap, const float* temp)
{
    const int cnt = min(*count, cap);
    const long long total = (long long)cnt * ncols;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % cnt);
        const long long c = idx / cnt;
        A[c * lda + tgt[i]] = temp[c * cap + i];
    }
}

}  // namespace

// Dynamic shared-memory opt-ins, set once per handle creation (never inside a
// stream capture).
void configure_getrf_kernels(hdbf_context* ctx)
{
    const size_t cap8 = ctx->max_smem_optin > 8192 ? ctx->max_smem_optin - 8192 : 40960;
    const size_t cap4 = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    cudaFuncSetAttribute(getf2_coop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap8);
    cudaFuncSetAttribute(compose_swaps_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap4);
    cudaFuncSetAttribute(compose_swaps_serial_kernel,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap4);
    cudaFuncSetAttribute(apply_moves_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap4);
    cudaFuncSetAttribute(compose_running_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap4);
    cudaGetLastError();
}

size_t getf2_coop_scratch_bytes()
{
    return align_up((size_t)(2 * kCoopMaxGrid * kSlotWords) * sizeof(unsigned long long), 256);
}

hdbf_status getf2_coop(hdbf_context* ctx, int m, int w, float* A, long long lda, int* ipiv,
                       int ipiv_add, int* info, int info_base, bool pivot)
{
    int piv_flag = pivot ? 1 : 0;
    if (m <= 0 || w <= 0) return HDBF_STATUS_SUCCESS;
    if (w > kCoopMaxW) return HDBF_STATUS_INVALID_VALUE;
    HDBF_TRY(ensure_ws(ctx, 64));
    unsigned long long* scr = reinterpret_cast<unsigned long long*>(ws_coop(ctx));

    // Grid: ~256 rows per CTA (panel_rows; measured fastest at n = 32768),
    // more when the slice would not fit in shared memory, at most one CTA per
    // SM; co-residency is guaranteed by the cooperative launch, which fails
    // instead of hanging if the grid cannot fit.
    const size_t smem_cap = ctx->max_smem_optin > 8192 ? ctx->max_smem_optin - 8192 : 40960;
    const size_t row_bytes = (size_t)w * sizeof(float);
    const long long fit_rows = (long long)(smem_cap / row_bytes);
    const int target = ctx->panel_rows > 0 ? ctx->panel_rows : 256;
    int G = (m + target - 1) / target;
    if (fit_rows > 0 && (m + fit_rows - 1) / fit_rows > G) G = (int)((m + fit_rows - 1) / fit_rows);
    if (G > ctx->sm_count) G = ctx->sm_count;
    if (G > kCoopMaxGrid) G = kCoopMaxGrid;
    if (G < 1) G = 1;
    int rpc = (m + G - 1) / G;
    size_t smem = (size_t)rpc * w * sizeof(float);
    if (smem > smem_cap || rpc >= (int)kNoRow) return HDBF_STATUS_NOT_SUPPORTED;
    unsigned* epoch = reinterpret_cast<unsigned*>(ctx->dev_small + kSmallEpoch);
    unsigned* done = reinterpret_cast<unsigned*>(ctx->dev_small + kSmallDone);
    int* err = ctx->dev_small + kSmallErr;
    ProfScope prof(ctx, kClsPanel, (double)m * w * w - (double)w * w * w / 3.0, 8.0 * m * w);
    void* args[] = {&m, &w, &A, &lda, &rpc, &ipiv, &ipiv_add, &info, &info_base,
                    &scr, &epoch, &done, &err, &piv_flag};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)getf2_coop_kernel, dim3(G),
                                                dim3(kCoopThreads), args, smem, ctx->stream);
    ctx->launches++;
    if (e != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    return HDBF_STATUS_SUCCESS;
}

hdbf_status compose_swaps(hdbf_context* ctx, const int* ipiv, int k, int ipiv_minus, int m,
                          int* src, int* tgt, int* count, int* gperm, int* info)
{
    if (k <= 0 || m <= 0) return HDBF_STATUS_SUCCESS;
    if (k > m) return HDBF_STATUS_INVALID_VALUE;
    const size_t cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    if (k <= kComposeMaxK) {
        const size_t smem = compose_sorted_bytes(0, k);
        ProfScope prof(ctx, kClsCompose, 0.0, 12.0 * k);
        compose_swaps_kernel<<<1, kComposeThreads, smem, ctx->stream>>>(
            ipiv, k, ipiv_minus, m, src, tgt, count, info, ctx->dev_small + kSmallErr);
        ctx->launches++;
        return last_cuda(ctx);
    }
    const size_t smem = (size_t)m * sizeof(int);
    const int use_smem = smem <= cap ? 1 : 0;
    if (!use_smem && !gperm) return HDBF_STATUS_INVALID_VALUE;
    ProfScope prof(ctx, kClsCompose, 0.0, 4.0 * k + 8.0 * m);
    compose_swaps_serial_kernel<<<1, kComposeThreads, use_smem ? smem : 0, ctx->stream>>>(
        ipiv, k, ipiv_minus, m, src, tgt, count, gperm, use_smem, info,
        ctx->dev_small + kSmallErr);
    ctx->launches++;
    return last_cuda(ctx);
}

bool compose_running_fits(hdbf_context* ctx, int m, int kk)
{
    const size_t cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    return kk >= 0 && kk <= kComposeMaxK && compose_sorted_bytes(m, kk) <= cap;
}

hdbf_status compose_running(hdbf_context* ctx, const int* ipiv, int k0, int k1, int ipiv_minus,
                            int m, int* pos, bool init, int* src, int* tgt, int* count, int* info)
{
    if (m <= 0) return HDBF_STATUS_SUCCESS;
    if (k0 < 0 || k1 < k0 || k1 > m || !compose_running_fits(ctx, m, k1 - k0))
        return HDBF_STATUS_INVALID_VALUE;
    ProfScope prof(ctx, kClsCompose, 0.0, 12.0 * (k1 - k0) + 12.0 * m);
    const size_t smem = compose_sorted_bytes(m, k1 - k0);
    compose_running_kernel<<<1, kComposeThreads, smem, ctx->stream>>>(
        ipiv, k0, k1, ipiv_minus, m, pos, init ? 1 : 0, src, tgt, count, info,
        ctx->dev_small + kSmallErr);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status apply_moves(hdbf_context* ctx, float* A, long long lda, int ncols,
                        const int* src, const int* tgt, const int* count, int max_moves,
                        float* temp, long long temp_cols)
{
    if (ncols <= 0 || max_moves <= 0) return HDBF_STATUS_SUCCESS;
    const size_t per_col = (size_t)max_moves * sizeof(float);
    const size_t idx_bytes = 2 * (size_t)max_moves * sizeof(int);
    const size_t budget = 64 * 1024;
    const size_t hard_cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    ProfScope prof(ctx, kClsMoves, 0.0, 8.0 * (double)max_moves * ncols);
    if (per_col + idx_bytes <= hard_cap) {
        int cpc = (int)((budget > idx_bytes ? budget - idx_bytes : 0) / per_col);
        if (cpc < 1) cpc = 1;
        if (cpc > 16) cpc = 16;
        const int grid = (ncols + cpc - 1) / cpc;
        apply_moves_smem_kernel<<<grid, kApplyThreads, per_col * cpc + idx_bytes, ctx->stream>>>(
            A, lda, ncols, src, tgt, count, cpc, max_moves);
        ctx->launches++;
        return last_cuda(ctx);
    }
    if (!temp || temp_cols <= 0) return HDBF_STATUS_INVALID_VALUE;
    for (long long c = 0; c < ncols; c += temp_cols) {
        const int nc = (int)((ncols - c) < temp_cols ? (ncols - c) : temp_cols);
        const long long total = (long long)nc * max_moves;
        const int grid = (int)((total + 255) / 256 < 65535 ? (total + 255) / 256 : 65535);
        gather_rows_kernel<<<grid, 256, 0, ctx->stream>>>(A + c * lda, lda, nc, src, count,
                                                          max_moves, temp);
        scatter_rows_kernel<<<grid, 256, 0, ctx->stream>>>(A + c * lda, lda, nc, tgt, count,
                                                           max_moves, temp);
        ctx->launches += 2;
    }
    return last_cuda(ctx);
}

}  // namespace hdbf
