// steady_ant.cu -- unit-Monge (sticky braid) multiplication R = P (.) Q on sm_100a.
//
// Same recursion as the reference's steady ant (R:common/include/Permutations/MongeMultuplicationStrategy.h:
// 487-593): split the common index into two halves, multiply the halves, map them back (inverseMapping
// :208-220) and combine them along the demarcation line (antPassage :244-301, restoreMatrixInRlo :304-323).
// The product is unique, so the tree of splits is free to choose; here it is the bottom-up tree of aligned
// power-of-two ranges of the common index, evaluated level by level:
//   * node J = [lo, hi) of the common index keeps PL = rows of P whose column lies in J (sorted), QL = columns
//     of Q whose row lies in J (sorted), and RES = the node's product in node-local coordinates;
//   * a leaf j has PL = {P^-1(j)}, QL = {Q(j)}, RES = {(0, 0)};
//   * merging the children is a merge of sorted lists (the positions are the reference's row/column mappers)
//     followed by the ant passage.
// The ant passage is restated data-parallel: for a node of size k with combined points (row r -> x_r, lo/hi)
//   delta(r, c) = #{hi points: row < r, col < c} - #{lo points: row >= r, col >= c}
// (the reference's rhi - rlo, BOTTOM_RIGHT / TOP_LEFT dominance sums, R:common/include/Permutations/
// DominanceSum.h:210-294), c*(r) = min{c : delta(r, c) >= 0}, and the product keeps x_r in row r except where
// 1 <= c*(r) <= k and the row's point lies on the wrong side of c*(r) (a hi point left of it or a lo point at
// or right of it): there the point moves to column c*(r) - 1 (the reference's "good points").  Row by row,
// c*(r) = c*(r+1) unless row r's point flips the sign, else one past the next column whose point raises
// delta(r, .).  c* at every 32nd row is found by warp-wide ballot scans.  Inside a CTA's shared-memory subtree (up
// to 2^12 common indices) the nodes of up to kNodeW leaves come straight from the product's definition as a
// 0-Hecke product, by a sorting network (warp_node); spans up to 512 walk the rows between the 32-row boundaries;
// from span 1024 those rows are not walked: c* is non-increasing in r and the product is a permutation, so the
// moving rows take exactly their own columns, the topmost row the largest, and a row moves iff the sign of
// delta(r, x_r) says so; that sign comes from the c* of the row's 32-row segment and two short counts.  At the
// HBM levels the rows between are walked by one thread (or, for a long column span, one warp) each.
#include <algorithm>
#include <climits>
#include <numeric>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

constexpr int kSaSB = 4096;      // largest subtree a CTA finishes in shared memory
constexpr int kSaThreads = 256;
constexpr int kSaSF = 32;        // rows per walk (fine band)
constexpr int kSaSC = 512;       // rows per coarse band (full-scan boundaries)
constexpr int kSaPerThread = kSaSB / kSaThreads;
constexpr int kSaRankSpan = 1024;  // node spans from which the moving rows are ranked instead of walked
constexpr int kSegW = kSaSB / 32 / (kSaThreads / 32);   // 32-row segments per warp in the rank passes
constexpr int kSegB = 8;                                  // segments whose loads a rank pass batches
static_assert(kSegW % kSegB == 0 && kSegB <= 32, "rank passes take whole batches");
constexpr int kNodeW = 128;      // leaves of the nodes the sorting network finishes (spans 2 .. kNodeW)
constexpr int kLowGroups = 1;   // such nodes a warp takes through the network at once
constexpr int kWalkSpanMax = 64;   // walks crossing more columns are taken by a whole warp

static_assert(kSaSB / kSaSF <= kSaThreads - 32, "the walk phase needs at least one warp without a thread walk");

struct SaBlockItem {
    int64_t off;   // first common index of the block (concatenated problem layout)
    int nb;        // block size (<= kSaSB)
    int pad;
};

struct SaShared {
    int32_t PL[kSaSB];
    int32_t QL[kSaSB];
    uint16_t RES[kSaSB];
    uint16_t posP[kSaSB];
    uint16_t posQ[kSaSB];
    uint16_t xs[kSaSB];   // node-local row -> col | hi << 15
    uint16_t ys[kSaSB];   // node-local col -> row | hi << 15
    int32_t cst[kSaSB / kSaSF + 8];    // c* at node row R, slot (node start + R) / kSaSF
    int32_t sub[kSaSB / kSaSC];        // lo rows per kSaSC-row sub-band of the block (coarse phase)
};

__device__ __forceinline__ int count_less(const int32_t *arr, int lo, int hi, int32_t v) {
    // number of entries < v in the sorted range arr[lo, hi)
    int l = lo, h = hi;
    while (l < h) {
        const int mid = (l + h) >> 1;
        if (arr[mid] < v) l = mid + 1;
        else h = mid;
    }
    return l - lo;
}

// warp-wide: one past the need-th g in [from, end) with pred(g), `none` when there are fewer.  U 32-wide
// chunks per round: their loads are independent, so a round costs about one load latency (U = 4 for scans that
// are usually long, 1 for the short ones).
template <int U, typename Pred>
__device__ __forceinline__ int ballot_search(int from, int end, int need, int none, int lane, Pred pred) {
    if (need <= 0) return from;
    for (int g0 = from; g0 < end; g0 += 32 * U) {
        bool q[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int g = g0 + 32 * u + lane;
            q[u] = g < end && pred(g);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const unsigned m = __ballot_sync(kFull, q[u]);
            const int cnt = __popc(m);
            if (need <= cnt) return g0 + 32 * u + (int) __fns(m, 0, need) + 1;
            need -= cnt;
        }
    }
    return none;
}

// warp-wide: the first i in [l, h) with pred(i), h when there is none (pred monotone: false ... true).  33-way
// rounds (one probe per lane), so a search over 2^22 entries takes four dependent loads instead of 22.
template <typename Pred>
__device__ __forceinline__ int warp_first_true(int l, int h, int lane, Pred pred) {
    while (h - l > 32) {
        const int mid = l + (int) (((int64_t) (h - l) * (lane + 1)) / 33);   // strictly increasing probes in [l, h)
        const int t = __popc(__ballot_sync(kFull, !pred(mid)));              // probes below the answer
        const int nl = t == 0 ? l : __shfl_sync(kFull, mid, t - 1) + 1;
        const int nh = t == 32 ? h : __shfl_sync(kFull, mid, t & 31);
        l = nl;
        h = nh;
    }
    const int i = l + lane;
    return l + __popc(__ballot_sync(kFull, i < h && !pred(i)));
}

// warp-wide: #{i in [i0, i1) : pred(i)}, U 32-wide chunks per round
template <int U, typename Pred>
__device__ __forceinline__ int ballot_count(int i0, int i1, int lane, Pred pred) {
    int total = 0;
    for (int b = i0; b < i1; b += 32 * U) {
        bool q[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = b + 32 * u + lane;
            q[u] = i < i1 && pred(i);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) total += __popc(__ballot_sync(kFull, q[u]));
    }
    return total;
}

// warp-wide: number of rows r in [r0, r1) of the node at base a whose point raises delta when moving up
// past it at column c (rowind(r, c) = hi ? x < c : x >= c)
template <int U = 1>
__device__ __forceinline__ int warp_row_count(const SaShared &S, int a, int r0, int r1, int c, int lane) {
    return ballot_count<U>(r0, r1, lane, [&](int r) {
        const int v = S.xs[a + r];
        const int x = v & 0x7fff;
        return (v >> 15) ? (x < c) : (x >= c);
    });
}

// warp-wide: one past the need-th column g >= from whose point raises delta in row R
// (colind(g, R) = hi ? y < R : y >= R); k + 1 when there is none
template <int U = 1>
__device__ __forceinline__ int warp_col_search(const SaShared &S, int a, int k, int from, int need, int R, int lane) {
    return ballot_search<U>(from, k, need, k + 1, lane, [&](int g) {
        const int w = S.ys[a + g];
        const int y = w & 0x7fff;
        return (w >> 15) ? (y < R) : (y >= R);
    });
}

// flat task index -> (node, task within node); full nodes have per_full tasks, the trailing node the rest
__device__ __forceinline__ void task_node(int t, int per_full, int nfull, int &nd, int &jj) {
    if (t < nfull * per_full) {
        nd = t / per_full;
        jj = t - nd * per_full;
    } else {
        nd = nfull;
        jj = t - nfull * per_full;
    }
}

// one thread: node-local parent positions of the outputs [d, d + cnt) of the merge of the sorted lists
// L[a, m) (lo child) and L[m, b) (hi child): a merge-path search for the split of the first d outputs, then a
// sequential merge (the reference's row / column mappers, R:common/include/Permutations/
// MongeMultuplicationStrategy.h:208-220, for every element of the two children)
__device__ __forceinline__ void merge_positions(const int32_t *L, int a, int m, int b, int d, int cnt,
                                                uint16_t *pos) {
    const int nlo = m - a, nhi = b - m;
    int l = max(0, d - nhi), h = min(d, nlo);
    while (l < h) {
        const int mid = (l + h) >> 1;
        if (L[a + mid] < L[m + d - 1 - mid]) l = mid + 1;
        else h = mid;
    }
    int i = l, j = d - l;
    int32_t vlo = i < nlo ? L[a + i] : INT_MAX;
    int32_t vhi = j < nhi ? L[m + j] : INT_MAX;
    for (int s = 0; s < cnt; ++s) {
        if (vlo < vhi) {
            pos[a + i] = (uint16_t) (d + s);
            ++i;
            vlo = i < nlo ? L[a + i] : INT_MAX;
        } else {
            pos[m + j] = (uint16_t) (d + s);
            ++j;
            vhi = j < nhi ? L[m + j] : INT_MAX;
        }
    }
}

// one thread: the walk of the kSaSF rows [top, bot) (top a multiple of kSaSF in the block, bot - top <= kSaSF,
// the rows past bot unused) with the rows' points held in registers and the products written back packed
__device__ __forceinline__ void thread_walk32(SaShared &S, int a, int k, int top, int bot, int c) {
    static_assert(kSaSF == 32, "register walk assumes 32-row walks");
    uint32_t w[16];
    const uint4 *src = reinterpret_cast<const uint4 *>(S.xs + a + top);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint4 u = src[q];
        w[4 * q] = u.x;
        w[4 * q + 1] = u.y;
        w[4 * q + 2] = u.z;
        w[4 * q + 3] = u.w;
    }
    uint32_t o[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) o[q] = 0u;
    const uint16_t *ys = S.ys + a;
#pragma unroll
    for (int i = 31; i >= 0; --i) {
        const int r = top + i;
        if (r < bot) {
            const int v = (int) ((w[i >> 1] >> ((i & 1) * 16)) & 0xffffu);
            const int xr = v & 0x7fff;
            const bool hi = v >> 15;
            if (hi ? (xr < c) : (xr >= c)) {
                // next column g >= c whose point raises delta in row r; two columns per step
                int g = c;
                for (;;) {
                    if (g >= k) break;
                    const int w0 = ys[g];
                    const int w1 = g + 1 < k ? ys[g + 1] : 0;
                    if ((w0 >> 15) ? ((w0 & 0x7fff) < r) : ((w0 & 0x7fff) >= r)) break;
                    if (g + 1 >= k) {
                        g = k;
                        break;
                    }
                    if ((w1 >> 15) ? ((w1 & 0x7fff) < r) : ((w1 & 0x7fff) >= r)) {
                        g += 1;
                        break;
                    }
                    g += 2;
                }
                c = g < k ? g + 1 : k + 1;
            }
            const bool good = c >= 1 && c <= k && (hi ? (xr < c) : (xr >= c));
            o[i >> 1] |= (uint32_t) (good ? c - 1 : xr) << ((i & 1) * 16);
        }
    }
    uint4 *dst = reinterpret_cast<uint4 *>(S.RES + a + top);
#pragma unroll
    for (int q = 0; q < 4; ++q) dst[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
}


// one warp: the walk of rows [top, bot) for a walk whose column span is long; rows without a jump are
// settled 32 at a time by a ballot, every jump is a ballot scan of the columns
__device__ __forceinline__ void warp_walk(SaShared &S, int a, int k, int top, int bot, int c, int lane) {
    int rb = bot;   // rows [rb, bot) are done
    while (rb > top) {
        const int r = rb - 1 - lane;
        int v = 0;
        bool ind = false;
        if (r >= top) {
            v = S.xs[a + r];
            const int x = v & 0x7fff;
            ind = (v >> 15) ? (x < c) : (x >= c);
        }
        const unsigned m = __ballot_sync(kFull, ind);
        const int j = m ? __ffs(m) - 1 : 32;   // lanes below j keep their point
        if (lane < j && r >= top) S.RES[a + r] = (uint16_t) (v & 0x7fff);
        if (j == 32) {
            rb -= 32;
            continue;
        }
        const int rj = rb - 1 - j;
        const int vj = __shfl_sync(kFull, v, j);
        c = warp_col_search(S, a, k, c, 1, rj, lane);
        const int xr = vj & 0x7fff;
        const bool good = c >= 1 && c <= k && ((vj >> 15) ? (xr < c) : (xr >= c));
        if (lane == 0) S.RES[a + rj] = (uint16_t) (good ? c - 1 : xr);
        rb = rj;
    }
    __syncwarp();
}

// One warp: the products of the (32 E)-leaf nodes at o, o + 32 E, ... (group j holds cnt[j] <= 32 E leaves, 0 for
// none), each straight from its definition instead of through the merge levels of spans 2 .. 32 E.  The sticky
// product of permutations is the product of the 0-Hecke monoid (Tiskin's seaweed monoid): with w = P^-1 of the
// node in one-line notation (position = common index, value = row), bubble-sorting w by adjacent swaps s_i of
// inversions gives P = s_i1 s_i2 ... in sorting order, and R = Q * s_i1 * s_i2 * ... where "* s_i" swaps
// positions i, i+1 of the sequence only if that adds an inversion (the combing cell's rule).  So an odd-even
// transposition sort of the rows over 32 E rounds (lane l holds positions E l .. E l + E - 1), that swaps the
// carried column ranks on each of its swaps where they are ascending, leaves in position i the i-th smallest row
// and the node-local column of its point.  Pads past cnt hold INT_MAX rows and never move.  The column ranks come
// from counting inside each half of the node and a binary search of the other half; the sorted column list is
// their scatter.  Only __syncwarp: the nodes belong to this warp alone.
template <int E, int NG>
__device__ __forceinline__ void warp_node(SaShared &S, int o, const int (&cnt)[NG], int lane) {
    static_assert(E >= 2 && E % 2 == 0, "pairs of positions inside a lane");
    constexpr int W = 32 * E;
    int u[NG][E], r[NG][E], q[NG][E];
#pragma unroll
    for (int j = 0; j < NG; ++j)
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = E * lane + e;
            const bool v = x < cnt[j];
            u[j][e] = v ? S.PL[o + W * j + x] : INT_MAX;
            q[j][e] = v ? S.QL[o + W * j + x] : INT_MAX;
            r[j][e] = 0;
        }
    // column ranks inside the node (the columns are distinct): inside the lane's half of the node (16 lanes) by
    // counting, plus the other half's columns below by a binary search of that half's sorted columns
    constexpr int H = W / 2;   // positions per half
    const int hb = lane & 16;  // first lane of this lane's half
#pragma unroll 2
    for (int t = 0; t < 16; ++t) {
#pragma unroll
        for (int j = 0; j < NG; ++j)
#pragma unroll
            for (int f = 0; f < E; ++f) {
                const int a = __shfl_sync(kFull, q[j][f], hb + t);
#pragma unroll
                for (int e = 0; e < E; ++e) r[j][e] += a < q[j][e];
            }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < NG; ++j)
#pragma unroll
        for (int e = 0; e < E; ++e)
            if (E * lane + e < cnt[j]) S.QL[o + W * j + (hb ? H : 0) + r[j][e]] = q[j][e];
    __syncwarp();
#pragma unroll
    for (int j = 0; j < NG; ++j) {
        const int other = hb ? 0 : H;   // the other half's first position
        const int nother = min(H, max(0, cnt[j] - other));
        const int32_t *arr = S.QL + o + W * j + other;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            int pos = 0;   // entries of arr[0, nother) below q
#pragma unroll
            for (int st = H; st > 0; st >>= 1)
                if (pos + st <= nother && arr[pos + st - 1] < q[j][e]) pos += st;
            r[j][e] += pos;
        }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < NG; ++j)
#pragma unroll
        for (int e = 0; e < E; ++e)
            if (E * lane + e < cnt[j]) S.QL[o + W * j + r[j][e]] = q[j][e];
    const bool has_next = lane < 31, has_prev = lane > 0;
#pragma unroll 2
    for (int t = 0; t < W / 2; ++t) {
        // even round: positions (2i, 2i + 1), inside the lane
#pragma unroll
        for (int j = 0; j < NG; ++j)
#pragma unroll
            for (int e = 0; e < E; e += 2) {
                const bool c = u[j][e] > u[j][e + 1];
                const int lo = min(u[j][e], u[j][e + 1]), hi = max(u[j][e], u[j][e + 1]);
                const int rmax = max(r[j][e], r[j][e + 1]), rmin = min(r[j][e], r[j][e + 1]);
                u[j][e] = lo;
                u[j][e + 1] = hi;
                r[j][e] = c ? rmax : r[j][e];
                r[j][e + 1] = c ? rmin : r[j][e + 1];
            }
        // odd round: positions (2i + 1, 2i + 2): inside the lane, and this lane's last with the next lane's first
#pragma unroll
        for (int j = 0; j < NG; ++j) {
            const int un = __shfl_down_sync(kFull, u[j][0], 1), rn = __shfl_down_sync(kFull, r[j][0], 1);
            const int up = __shfl_up_sync(kFull, u[j][E - 1], 1), rp = __shfl_up_sync(kFull, r[j][E - 1], 1);
#pragma unroll
            for (int e = 1; e + 1 < E; e += 2) {
                const bool c = u[j][e] > u[j][e + 1];
                const int lo = min(u[j][e], u[j][e + 1]), hi = max(u[j][e], u[j][e + 1]);
                const int rmax = max(r[j][e], r[j][e + 1]), rmin = min(r[j][e], r[j][e + 1]);
                u[j][e] = lo;
                u[j][e + 1] = hi;
                r[j][e] = c ? rmax : r[j][e];
                r[j][e + 1] = c ? rmin : r[j][e + 1];
            }
            const bool c1 = has_next && u[j][E - 1] > un;
            const bool c0 = has_prev && up > u[j][0];
            r[j][E - 1] = c1 ? max(r[j][E - 1], rn) : r[j][E - 1];
            u[j][E - 1] = c1 ? un : u[j][E - 1];
            r[j][0] = c0 ? min(rp, r[j][0]) : r[j][0];
            u[j][0] = c0 ? up : u[j][0];
        }
    }
#pragma unroll
    for (int j = 0; j < NG; ++j)
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = E * lane + e;
            if (x < cnt[j]) {
                S.PL[o + W * j + x] = u[j][e];
                S.RES[o + W * j + x] = (uint16_t) r[j][e];
            }
        }
    __syncwarp();
}

__global__ void __launch_bounds__(kSaThreads, 3) sa_block_kernel(const int32_t *__restrict__ Pinv,
                                                             const int32_t *__restrict__ Q,
                                                             const SaBlockItem *__restrict__ items,
                                                             int32_t *__restrict__ PLout, int32_t *__restrict__ QLout,
                                                             int32_t *__restrict__ RESout, int *err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SaShared &S = *reinterpret_cast<SaShared *>(smem_raw);
    const SaBlockItem it = items[blockIdx.x];
    const int nb = it.nb;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = kSaThreads / 32;
    for (int e = tid; e < nb; e += kSaThreads) {
        S.PL[e] = Pinv[it.off + e];
        S.QL[e] = Q[it.off + e];
        S.RES[e] = 0;
    }
    __syncthreads();
    // spans 2 .. kNodeW: one warp per kNodeW-leaf node, the product by a sorting network
    for (int o = warp * kNodeW * kLowGroups; o < nb; o += nwarps * kNodeW * kLowGroups) {
        int cnt[kLowGroups];
#pragma unroll
        for (int j = 0; j < kLowGroups; ++j) cnt[j] = max(0, min(kNodeW, nb - o - kNodeW * j));
        warp_node<kNodeW / 32, kLowGroups>(S, o, cnt, lane);
    }
    __syncthreads();
    for (int size = kNodeW; size < nb; size <<= 1) {
        const int span = size << 1;
        // ---- merge the children's lists: positions in the parent lists ----
        if (span >= 2 * kSaPerThread) {
            // kSaPerThread consecutive outputs per thread (all inside one node: nodes are aligned multiples)
            const int o = tid * kSaPerThread;
            if (o < nb) {
                const int a = o & ~(span - 1);
                const int m = min(a + size, nb), b = min(a + span, nb);
                const int cnt = min(kSaPerThread, b - o);
                if (m >= b) {
                    for (int x = 0; x < cnt; ++x) S.posP[o + x] = S.posQ[o + x] = (uint16_t) (o + x - a);
                } else {
                    merge_positions(S.PL, a, m, b, o - a, cnt, S.posP);
                    merge_positions(S.QL, a, m, b, o - a, cnt, S.posQ);
                }
            }
        } else
        for (int e = tid; e < nb; e += kSaThreads) {
            const int a = e & ~(span - 1);
            const int m = min(a + size, nb), b = min(a + span, nb);
            int pp, pq;
            if (m >= b) {
                pp = pq = e - a;
            } else if (e < m) {
                pp = (e - a) + count_less(S.PL, m, b, S.PL[e]);
                pq = (e - a) + count_less(S.QL, m, b, S.QL[e]);
            } else {
                pp = (e - m) + count_less(S.PL, a, m, S.PL[e]);
                pq = (e - m) + count_less(S.QL, a, m, S.QL[e]);
            }
            S.posP[e] = (uint16_t) pp;
            S.posQ[e] = (uint16_t) pq;
        }
        __syncthreads();
        // ---- children's products in the parent's coordinates (inverse mapping) ----
        for (int e = tid; e < nb; e += kSaThreads) {
            const int a = e & ~(span - 1);
            const int m = min(a + size, nb), b = min(a + span, nb);
            if (m >= b) continue;
            const bool hi = e >= m;
            const int cs = hi ? m : a;
            const int rc = S.RES[e];
            if (rc >= (hi ? b - m : m - a)) {   // never expected: report, keep shared accesses in bounds
                raise_error(err, kDevErrBadState);
                continue;
            }
            const int row = S.posP[e];
            const int col = S.posQ[cs + rc];
            if (row >= b - a || col >= b - a) {   // positions of an inconsistent merge: report, stay in bounds
                raise_error(err, kDevErrBadState);
                continue;
            }
            S.xs[a + row] = (uint16_t) (col | (hi ? 0x8000 : 0));
            S.ys[a + col] = (uint16_t) (row | (hi ? 0x8000 : 0));
        }
        // ---- reorder the lists in place (values staged in registers, one list at a time) ----
        int32_t v[kSaPerThread];
#pragma unroll
        for (int i = 0; i < kSaPerThread; ++i) {
            const int e = tid + i * kSaThreads;
            if (e < nb) v[i] = S.PL[e];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kSaPerThread; ++i) {
            const int e = tid + i * kSaThreads;
            if (e < nb) S.PL[(e & ~(span - 1)) + S.posP[e]] = v[i];
        }
#pragma unroll
        for (int i = 0; i < kSaPerThread; ++i) {
            const int e = tid + i * kSaThreads;
            if (e < nb) v[i] = S.QL[e];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kSaPerThread; ++i) {
            const int e = tid + i * kSaThreads;
            if (e < nb) S.QL[(e & ~(span - 1)) + S.posQ[e]] = v[i];
        }
        __syncthreads();
        // ---- ant passage for every node of this level that has two children ----
        const int nfull = nb / span;                  // nodes of size span
        const int rem = nb - nfull * span;            // size of the trailing node
        if (span > kSaSF) {
            // phase A: coarse boundaries (multiples of kSaSC inside each node).  c*(R) is the need-th column
            // raising delta in row R, need = the lo rows at or below R: counted once per kSaSC-row sub-band (warp
            // w: block rows [w kSaSC, (w+1) kSaSC), inside one node) and summed per boundary.
            if (warp * kSaSC < nb) {
                const int r0 = warp * kSaSC, r1 = min(r0 + kSaSC, nb);
                const int cnt = ballot_count<4>(r0, r1, lane, [&](int r) { return !(S.xs[r] >> 15); });
                if (lane == 0) S.sub[warp] = cnt;
            }
            __syncthreads();
            const int ca_full = (span - 1) / kSaSC;
            const int ca_last = rem > size ? (rem - 1) / kSaSC : 0;
            for (int t = warp; t < nfull * ca_full + ca_last; t += nwarps) {
                int nd, jj;
                task_node(t, ca_full, nfull, nd, jj);
                const int a = nd * span, k = nd < nfull ? span : rem;
                const int R = (jj + 1) * kSaSC;
                int need = 0;   // lo rows at or below R
                for (int w = (a + R) / kSaSC; w * kSaSC < a + k; ++w) need += S.sub[w];
                const int cst = warp_col_search<4>(S, a, k, 0, need, R, lane);
                if (lane == 0) S.cst[(a + R) / kSaSF] = cst;
            }
            __syncthreads();
            // phase B: c* at every multiple of kSaSF (row 0 included) inside each sub-band of min(span, kSaSC)
            // rows, bottom-up from the boundary below the sub-band
            const int sb = span < kSaSC ? span : kSaSC;
            const int sb_full = span / sb;
            const int sb_last = rem > size ? (rem + sb - 1) / sb : 0;
            for (int t = warp; t < nfull * sb_full + sb_last; t += nwarps) {
                int nd, jj;
                task_node(t, sb_full, nfull, nd, jj);
                const int a = nd * span, k = nd < nfull ? span : rem;
                const int top = jj * sb, bot = min(top + sb, k);
                int cb = bot >= k ? 0 : S.cst[(a + bot) / kSaSF];
                const int Rlo = top == 0 ? 0 : top + kSaSF;
                for (int R = ((bot - 1) / kSaSF) * kSaSF; R >= Rlo; R -= kSaSF) {
                    const int Rn = min(R + kSaSF, bot);
                    int cst = k + 1;
                    if (cb <= k) {
                        const int need = warp_row_count(S, a, R, Rn, cb, lane);
                        cst = warp_col_search(S, a, k, cb, need, R, lane);
                    }
                    if (lane == 0) S.cst[(a + R) / kSaSF] = cst;
                    cb = cst;
                }
            }
            __syncthreads();
            if (span < kSaRankSpan) {
                // phase C: walks of kSaSF rows, each from the c* of its bottom boundary.  The first warps walk one
                // row band per thread; walks with a long column span are left to the remaining warps, which take
                // them one whole warp each at the same time
                const int wb_full = span / kSaSF;
                const int wb_last = rem > size ? (rem + kSaSF - 1) / kSaSF : 0;
                const int W = nfull * wb_full + wb_last;
                const int nww = (W + 31) >> 5;
                auto walk_of = [&](int t, int &a, int &k, int &top, int &bot) {
                    int nd, jj;
                    task_node(t, wb_full, nfull, nd, jj);
                    a = nd * span;
                    k = nd < nfull ? span : rem;
                    top = jj * kSaSF;
                    bot = min(top + kSaSF, k);
                };
                auto is_long = [&](int a, int k, int top, int bot) {
                    const int c = bot >= k ? 0 : S.cst[(a + bot) / kSaSF];
                    const int ce = S.cst[(a + top) / kSaSF];
                    return min(ce, k) - min(c, k) > kWalkSpanMax;
                };
                if (warp < nww) {
                    if (tid < W) {
                        int a, k, top, bot;
                        walk_of(tid, a, k, top, bot);
                        if (!is_long(a, k, top, bot))
                            thread_walk32(S, a, k, top, bot, bot >= k ? 0 : S.cst[(a + bot) / kSaSF]);
                    }
                } else {
                    const int h = warp - nww, nh = nwarps - nww;
                    int seen = 0;
                    for (int t0 = 0; t0 < W; t0 += 32) {
                        bool lng = false;
                        if (t0 + lane < W) {
                            int a, k, top, bot;
                            walk_of(t0 + lane, a, k, top, bot);
                            lng = is_long(a, k, top, bot);
                        }
                        unsigned msk = __ballot_sync(kFull, lng);
                        while (msk) {
                            const int l = __ffs(msk) - 1;
                            msk &= msk - 1;
                            if (seen % nh == h) {
                                int a, k, top, bot;
                                walk_of(t0 + l, a, k, top, bot);
                                warp_walk(S, a, k, top, bot, bot >= k ? 0 : S.cst[(a + bot) / kSaSF], lane);
                            }
                            ++seen;
                        }
                    }
                }
            } else {
            // phase C: the rows whose point moves.  c*(r) is non-increasing in r and the product is a permutation,
            // so the moving rows of a node take exactly their own columns, the topmost row the largest: a row moves
            // iff delta(r, x_r) puts its point on the wrong side of c*(r) (hi: delta < 0, lo: delta >= 0), and the
            // j-th moving row from the top takes the j-th largest of the moving rows' columns.  In the 32-row
            // segment [R, bot) of row r, with cb = c*(bot) (where delta(bot, cb) = 0),
            //   delta(r, x) = #{g in [cb, x): colind(g, bot)} - #{r' in [r, bot): rowind(r', x)},
            // and a row with x < cb (delta < 0) or x >= c*(R) (delta >= 0) needs no count at all.
            uint32_t *gbits = reinterpret_cast<uint32_t *>(S.posQ);   // moving rows, one bit per row
            uint32_t *cbits = gbits + kSaSB / 32;                     // moving columns, one bit per column
            int32_t *gpre = reinterpret_cast<int32_t *>(cbits + kSaSB / 32);   // exclusive prefixes of the words
            int32_t *cpre = gpre + kSaSB / 32 + 1;
            uint16_t *byrank = S.posP;                                // moving columns by descending rank
            const int cov = nfull * span + (rem > size ? rem : 0);   // rows of the nodes with two children
            const int nseg = (cov + 31) >> 5;
            // Segments sg = warp + i nwarps, kSegB at a time: every load of a batch is issued before its results
            // are used, and a segment's words are loaded by lane i and broadcast by shuffles.  Segment sg covers
            // block rows [32 sg, 32 sg + 32), so its top's c* is cst[sg] and its bottom's cst[sg + 1] (0 at the
            // bottom of the node).
            for (int b0 = 0; b0 < kSegW; b0 += kSegB) {
                int vv[kSegB];
#pragma unroll
                for (int i = 0; i < kSegB; ++i) {
                    const int row = ((warp + (b0 + i) * nwarps) << 5) + lane;
                    vv[i] = row < cov ? S.xs[row] : 0;
                }
                int ce_l = 0, cb_l = 0;
                {
                    const int sg = warp + (b0 + (lane & (kSegB - 1))) * nwarps;
                    if (sg < nseg) {
                        const int a = (sg << 5) & ~(span - 1);
                        const int k = a < nfull * span ? span : rem;
                        ce_l = S.cst[sg];
                        cb_l = (sg << 5) - a + 32 >= k ? 0 : S.cst[sg + 1];
                    }
                }
#pragma unroll
                for (int i = 0; i < kSegB; ++i) {
                    const int sg = warp + (b0 + i) * nwarps;
                    if (sg >= nseg) break;
                    const int a = (sg << 5) & ~(span - 1);
                    const int k = a < nfull * span ? span : rem;
                    const int R = (sg << 5) - a, bot = min(R + 32, k);
                    const int ce = __shfl_sync(kFull, ce_l, i), cb = __shfl_sync(kFull, cb_l, i);
                    const bool valid = R + lane < k;
                    const int v = vv[i];
                    const int x = v & 0x7fff;
                    const bool hi = v >> 15;
                    bool good = x < cb ? hi : !hi;
                    const bool hard = valid && x >= cb && x < ce;
                    const unsigned hm = __ballot_sync(kFull, hard);
                    if (hm) {
                        int t2 = 0;   // rows [r, bot) whose point raises delta when moving up past them at column x
                        for (unsigned rest = hm; rest; rest &= rest - 1) {
                            const int hl = __ffs(rest) - 1;
                            const int xh = __shfl_sync(kFull, x, hl);
                            const unsigned mk =
                                __ballot_sync(kFull, lane >= hl && R + lane < bot && (hi ? (x < xh) : (x >= xh)));
                            if (lane == hl) t2 = __popc(mk);
                        }
                        const int xmax = (int) __reduce_max_sync(kFull, hard ? (unsigned) x : 0u);
                        int t1 = 0;   // columns [cb, x) whose point raises delta in row bot
                        for (int g0 = cb; g0 < xmax; g0 += 32) {
                            const int g = g0 + lane;
                            bool q = false;
                            if (g < xmax) {
                                const int w = S.ys[a + g];
                                const int y = w & 0x7fff;
                                q = (w >> 15) ? (y < bot) : (y >= bot);
                            }
                            const unsigned mk = __ballot_sync(kFull, q);
                            if (x >= g0 + 32) t1 += __popc(mk);
                            else if (x > g0) t1 += __popc(mk & ((1u << (x - g0)) - 1u));
                        }
                        if (hard) good = hi ? (t1 - t2 < 0) : (t1 - t2 >= 0);
                    }
                    const unsigned gm = __ballot_sync(kFull, valid && good);
                    if (lane == 0) gbits[sg] = gm;
                    if (valid && !good) S.RES[(sg << 5) + lane] = (uint16_t) x;   // a point that stays
                }
            }
            __syncthreads();
            // a column moves with the row that owns it
            for (int b0 = 0; b0 < kSegW; b0 += kSegB) {
                int yy[kSegB];
#pragma unroll
                for (int i = 0; i < kSegB; ++i) {
                    const int col = ((warp + (b0 + i) * nwarps) << 5) + lane;
                    yy[i] = col < cov ? (col & ~(span - 1)) + (S.ys[col] & 0x7fff) : -1;
                }
                uint32_t gw[kSegB];
#pragma unroll
                for (int i = 0; i < kSegB; ++i) gw[i] = yy[i] >= 0 ? gbits[yy[i] >> 5] >> (yy[i] & 31) : 0u;
#pragma unroll
                for (int i = 0; i < kSegB; ++i) {
                    const int sg = warp + (b0 + i) * nwarps;
                    const unsigned m = __ballot_sync(kFull, gw[i] & 1u);
                    if (lane == 0 && sg < nseg) cbits[sg] = m;
                }
            }
            __syncthreads();
            if (warp < 2) {   // exclusive prefix counts of the row words (warp 0) and column words (warp 1)
                const uint32_t *bits = warp == 0 ? gbits : cbits;
                int32_t *pre = warp == 0 ? gpre : cpre;
                int loc[kSaSB / 1024];
                int sum = 0;
#pragma unroll
                for (int i = 0; i < kSaSB / 1024; ++i) {
                    const int w = lane * (kSaSB / 1024) + i;
                    loc[i] = w < nseg ? __popc(bits[w]) : 0;
                    sum += loc[i];
                }
                int inc = sum;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int t = __shfl_up_sync(kFull, inc, d);
                    if (lane >= d) inc += t;
                }
                int run = inc - sum;
#pragma unroll
                for (int i = 0; i < kSaSB / 1024; ++i) {
                    const int w = lane * (kSaSB / 1024) + i;
                    if (w < nseg) pre[w] = run;
                    run += loc[i];
                }
                if (lane == 31) pre[nseg] = inc;
            }
            __syncthreads();
            // moving columns by descending rank within the node
            for (int b0 = 0; b0 < kSegW; b0 += kSegB) {
                uint32_t cw_l = 0;
                int p_l = 0, ps_l = 0, pe_l = 0;
                {
                    const int sg = warp + (b0 + (lane & (kSegB - 1))) * nwarps;
                    if (sg < nseg) {
                        const int a = (sg << 5) & ~(span - 1);
                        const int k = a < nfull * span ? span : rem;
                        cw_l = cbits[sg];
                        p_l = cpre[sg];
                        ps_l = cpre[a >> 5];
                        pe_l = cpre[(a + k + 31) >> 5];
                    }
                }
#pragma unroll
                for (int i = 0; i < kSegB; ++i) {
                    const int sg = warp + (b0 + i) * nwarps;
                    if (sg >= nseg) break;
                    const uint32_t cw = __shfl_sync(kFull, cw_l, i);
                    const int p = __shfl_sync(kFull, p_l, i), ps = __shfl_sync(kFull, ps_l, i),
                              pe = __shfl_sync(kFull, pe_l, i);
                    if ((cw >> lane) & 1u) {
                        const int col = (sg << 5) + lane, a = col & ~(span - 1);
                        const int incl = p - ps + __popc(cw & ((2u << lane) - 1u));
                        byrank[a + (pe - ps) - incl] = (uint16_t) (col - a);
                    }
                }
            }
            __syncthreads();
            // the moving rows, the j-th from the top of its node taking the j-th largest moving column
            for (int b0 = 0; b0 < kSegW; b0 += kSegB) {
                uint32_t gw_l = 0;
                int p_l = 0, ps_l = 0;
                {
                    const int sg = warp + (b0 + (lane & (kSegB - 1))) * nwarps;
                    if (sg < nseg) {
                        gw_l = gbits[sg];
                        p_l = gpre[sg];
                        ps_l = gpre[((sg << 5) & ~(span - 1)) >> 5];
                    }
                }
                uint16_t val[kSegB];
#pragma unroll
                for (int i = 0; i < kSegB; ++i) {
                    const uint32_t gw = __shfl_sync(kFull, gw_l, i);
                    const int p = __shfl_sync(kFull, p_l, i), ps = __shfl_sync(kFull, ps_l, i);
                    const int a = ((warp + (b0 + i) * nwarps) << 5) & ~(span - 1);
                    val[i] = ((gw >> lane) & 1u) ? byrank[a + p - ps + __popc(gw & ((1u << lane) - 1u))] : 0;
                }
#pragma unroll
                for (int i = 0; i < kSegB; ++i) {
                    const uint32_t gw = __shfl_sync(kFull, gw_l, i);
                    if ((gw >> lane) & 1u) S.RES[((warp + (b0 + i) * nwarps) << 5) + lane] = val[i];
                }
            }
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < nb; e += kSaThreads) {
        PLout[it.off + e] = S.PL[e];
        QLout[it.off + e] = S.QL[e];
        RESout[it.off + e] = S.RES[e];
    }
}

// ------------------------------------------------------------------------------------------------------
// Levels above the shared-memory block: nodes of k > kSaSB common indices, held in global memory.
// ------------------------------------------------------------------------------------------------------
constexpr int kMT = 2048;        // merge tile (output elements per CTA)
constexpr int kBand = 4096;      // rows per band CTA at HBM levels (a multiple of every coarse block Sc <= 4096)
constexpr int kBandThreads = 256;
constexpr int kBandSub = kBand / (kBandThreads / 32);   // rows per warp sub-band
constexpr int kBandWalk = kBand / kBandThreads;         // rows per thread walk
constexpr int kBandYCap = 12288;   // columns a band stages in shared memory
// block table of a wider band, in the same space: 2 + 4 bytes per block and 2 per own row (kBand rows)
constexpr int kWideMaxBlocks = (4 * kBandYCap - 2 * 4096 - 2) / 6;
constexpr unsigned kHiBit = 1u << 30;
constexpr int kRowHistSmemMax = 200 * 1024;   // block-table width limit of sa_rowhist_kernel's histogram
constexpr int kValMask = (1 << 30) - 1;

struct SaNode {
    int64_t off;       // first common index of the node
    int k;             // node size
    int h;             // size of the lo child (k - h = hi child)
    int Sc;            // columns per table column block (a power of two)
    int G;             // table column blocks: ceil(k / Sc)
    int Sr;            // rows per table row block: max(Sc, kBand), so every band boundary that is a multiple of Sr
                       // is a table row
    int NR;            // table row blocks: ceil(k / Sr)
    int64_t tab_off;   // offset of the node's (NR+1) x (G+1) prefix table
    int64_t vec_off;   // offset of the node's lo-row prefix (NR+1 entries) and lo-col prefix (G+1 entries)
    int64_t cst_off;   // offset of the node's c* slots, one per band (row b kBand)
};

struct SaTile {
    int node;
    int t;      // tile index inside the node
};

// Merge-path splits of every merge tile's first output, of the row-id lists (.x) and the column-id lists (.y):
// one warp per tile and list (33-way search), so no merge CTA starts with a serial search of global memory.
__global__ void __launch_bounds__(256) sa_split_kernel(const SaNode *__restrict__ nodes, const SaTile *__restrict__ tiles,
                                                       int ntiles, const int32_t *__restrict__ PL,
                                                       const int32_t *__restrict__ QL, int2 *__restrict__ splits) {
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (w >= 2 * ntiles) return;
    const int t = w >> 1, which = w & 1;
    const SaTile tl = tiles[t];
    const SaNode nd = nodes[tl.node];
    const int nhi = nd.k - nd.h, o0 = tl.t * kMT;
    const int32_t *lo = (which ? QL : PL) + nd.off, *hi = lo + nd.h;
    // the merge path's split at diagonal o0: the first i with lo[i] >= hi[o0 - 1 - i]
    const int i = warp_first_true(max(0, o0 - nhi), min(o0, nd.h), lane,
                                  [&](int m) { return __ldg(lo + m) >= __ldg(hi + o0 - 1 - m); });
    if (lane == 0) reinterpret_cast<int *>(splits)[2 * t + which] = i;
}

// Merge the children's sorted lists of every node; pos receives the node-local parent position of every
// child element (the reference's row / column mappers).  blockIdx.y = 0: row-id lists (splits .x), 1: column-id
// lists.  A CTA stages its tile's two runs in shared memory; each thread finds its own merge-path split of the
// tile (a binary search) and merges kMerPT consecutive outputs sequentially; outputs and positions go out
// through shared memory in coalesced stores.  The ids in a node are distinct, so the merge has no ties.
constexpr int kMerPT = kMT / 256;
__global__ void __launch_bounds__(256) sa_merge_kernel(const SaNode *__restrict__ nodes, const SaTile *__restrict__ tiles,
                                                       const int2 *__restrict__ splits,
                                                       const int32_t *__restrict__ PLin, int32_t *__restrict__ PLout,
                                                       int32_t *__restrict__ posP, const int32_t *__restrict__ QLin,
                                                       int32_t *__restrict__ QLout, int32_t *__restrict__ posQ) {
    __shared__ int32_t sm[kMT];     // the lo run [0, na), then the hi run [na, na + nbb)
    __shared__ int32_t sout[kMT];   // merged values
    __shared__ int32_t spos[kMT];   // parent positions of the lo run, then of the hi run
    const int which = blockIdx.y;
    const int32_t *__restrict__ Lin = which ? QLin : PLin;
    int32_t *__restrict__ Lout = which ? QLout : PLout;
    int32_t *__restrict__ pos = which ? posQ : posP;
    const SaTile tl = tiles[blockIdx.x];
    const SaNode nd = nodes[tl.node];
    const int nlo = nd.h;
    const int o0 = tl.t * kMT, o1 = min(o0 + kMT, nd.k);
    const int2 s0 = splits[blockIdx.x];
    int i1 = nlo;   // the node's last tile ends with both lists consumed
    if (o1 < nd.k) {
        const int2 s1 = splits[blockIdx.x + 1];   // the next tile of the same node
        i1 = which ? s1.y : s1.x;
    }
    const int32_t *lo = Lin + nd.off, *hi = Lin + nd.off + nd.h;
    const int i0 = which ? s0.y : s0.x, j0 = o0 - i0, j1 = o1 - i1;
    const int na = i1 - i0, nbb = j1 - j0, tot = na + nbb;
    {   // the two runs: all of a thread's loads are issued before any of them is used (one load latency per CTA)
        int v[kMerPT];
#pragma unroll
        for (int u = 0; u < kMerPT; ++u) {
            const int x = threadIdx.x + 256 * u;
            v[u] = x < na ? lo[i0 + x] : (x < tot ? hi[j0 + x - na] : 0);
        }
#pragma unroll
        for (int u = 0; u < kMerPT; ++u) {
            const int x = threadIdx.x + 256 * u;
            if (x < tot) sm[x] = v[u];
        }
    }
    __syncthreads();
    const int d0 = threadIdx.x * kMerPT;
    if (d0 < tot) {
        int l = max(0, d0 - nbb), h = min(d0, na);   // the first i with lo[i] >= hi[d0 - 1 - i]
        while (l < h) {
            const int mid = (l + h) >> 1;
            if (sm[mid] < sm[na + d0 - 1 - mid]) l = mid + 1;
            else h = mid;
        }
        int i = l, j = d0 - l;
        int vlo = i < na ? sm[i] : INT_MAX, vhi = j < nbb ? sm[na + j] : INT_MAX;
        const int cnt = min(kMerPT, tot - d0);
#pragma unroll
        for (int t = 0; t < kMerPT; ++t) {
            if (t < cnt) {
                const bool take_lo = vlo < vhi;
                sout[d0 + t] = take_lo ? vlo : vhi;
                spos[take_lo ? i : na + j] = o0 + d0 + t;
                if (take_lo) {
                    ++i;
                    vlo = i < na ? sm[i] : INT_MAX;
                } else {
                    ++j;
                    vhi = j < nbb ? sm[na + j] : INT_MAX;
                }
            }
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < tot; x += blockDim.x) Lout[nd.off + o0 + x] = sout[x];
    for (int x = threadIdx.x; x < na; x += blockDim.x) pos[nd.off + i0 + x] = spos[x];
    for (int x = threadIdx.x; x < nbb; x += blockDim.x) pos[nd.off + nd.h + j0 + x] = spos[na + x];
}

// Children's products in the parent's coordinates: xs (row -> col | hi) and ys (col -> row | hi).
__global__ void __launch_bounds__(256) sa_map_kernel(const SaNode *__restrict__ nodes, const SaTile *__restrict__ tiles,
                                                     const int32_t *__restrict__ posP, const int32_t *__restrict__ posQ,
                                                     const int32_t *__restrict__ RES, int32_t *__restrict__ xs,
                                                     int32_t *__restrict__ ys, int *err) {
    // 256 threads, kMT / 256 elements each; every round of loads is issued before its values are used
    constexpr int U = kMT / 256;
    const SaTile tl = tiles[blockIdx.x];
    const SaNode nd = nodes[tl.node];
    const int e0 = tl.t * kMT, e1 = min(e0 + kMT, nd.k);
    int rc[U], row[U], col[U];
    bool ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int e = e0 + threadIdx.x + 256 * u;
        ok[u] = e < e1;
        rc[u] = ok[u] ? RES[nd.off + e] : 0;
        row[u] = ok[u] ? posP[nd.off + e] : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int e = e0 + threadIdx.x + 256 * u;
        const bool hi = e >= nd.h;
        if (ok[u] && (rc[u] < 0 || rc[u] >= (hi ? nd.k - nd.h : nd.h))) {
            raise_error(err, kDevErrBadState);
            ok[u] = false;
        }
        col[u] = ok[u] ? posQ[nd.off + (hi ? nd.h : 0) + rc[u]] : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        if (!ok[u]) continue;
        const bool hi = e0 + (int) threadIdx.x + 256 * u >= nd.h;
        xs[nd.off + row[u]] = col[u] | (hi ? kHiBit : 0);
        ys[nd.off + col[u]] = row[u] | (hi ? kHiBit : 0);
    }
}

// number of entries < v in the increasing sequence a[0, n)
__device__ __forceinline__ int lower_bound_g(const int32_t *__restrict__ a, int n, int v) {
    int l = 0, h = n;
    while (l < h) {
        const int mid = (l + h) >> 1;
        if (__ldg(a + mid) < v) l = mid + 1;
        else h = mid;
    }
    return l;
}

// Row g of a node's block table (one CTA per row block of Sr rows, g = 0..NR): the signed counts of the row
// block's points by column block (hi +1, lo -1) in a shared histogram, scanned along the columns (exclusive)
// into the table; row NR is all zeros (the column scan's total row).  The lo-row prefix (entry g) and the lo-col
// prefix (entries h = g mod (NR+1)) come from binary searches: the lo child's rows and columns in the parent
// are its merge positions, two increasing sequences, so the lo rows (columns) before a bound are a search.
__global__ void __launch_bounds__(256) sa_rowhist_kernel(const SaNode *__restrict__ nodes, const int2 *__restrict__ tasks,
                                                         const int32_t *__restrict__ xs, const int32_t *__restrict__ posP,
                                                         const int32_t *__restrict__ posQ, int32_t *__restrict__ tab,
                                                         int32_t *__restrict__ vec) {
    extern __shared__ int32_t hist[];   // G + 1 counters
    __shared__ int32_t warp_sums[8];
    __shared__ int32_t carry;
    const int2 tk = tasks[blockIdx.x];   // (node, row block)
    const SaNode nd = nodes[tk.x];
    const int W = nd.G + 1, g = tk.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int h = threadIdx.x; h < W; h += blockDim.x) hist[h] = 0;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1)
        vec[nd.vec_off + g] = lower_bound_g(posP + nd.off, nd.h, (int) min((int64_t) g * nd.Sr, (int64_t) INT_MAX));
    for (int h = g + (int) threadIdx.x * (nd.NR + 1); h < W; h += (int) blockDim.x * (nd.NR + 1))
        vec[nd.vec_off + nd.NR + 1 + h] = lower_bound_g(posQ + nd.off, nd.h, (int) min((int64_t) h * nd.Sc, (int64_t) INT_MAX));
    if (g < nd.NR) {
        const int r0 = g * nd.Sr, r1 = min(r0 + nd.Sr, nd.k);
        for (int rb = r0; rb < r1; rb += 8 * (int) blockDim.x) {   // eight loads in flight per thread
            int v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int r = rb + (int) threadIdx.x + (int) blockDim.x * u;
                v[u] = r < r1 ? xs[nd.off + r] : -1;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (v[u] < 0) continue;
                const int hh = (v[u] & kValMask) / nd.Sc;
                if (hh < W) atomicAdd(&hist[hh], (v[u] & kHiBit) ? 1 : -1);
            }
        }
    }
    __syncthreads();
    int32_t *row = tab + nd.tab_off + (int64_t) g * W;
    for (int c0 = 0; c0 < W; c0 += blockDim.x) {
        const int c = c0 + threadIdx.x;
        const int v = c < W ? hist[c] : 0;
        int incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += o;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        int woff = 0;
        for (int w = 0; w < warp; ++w) woff += warp_sums[w];
        const int excl = carry + woff + incl - v;
        __syncthreads();
        if (c < W) row[c] = excl;
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
}

// Exclusive prefix sums along g (the NR+1 table rows) of 32 table columns per block (lanes = columns, so every
// row access is one coalesced segment); the kScanColWarps warps take consecutive row ranges and combine their
// column totals.
constexpr int kScanColWarps = 32;
__global__ void __launch_bounds__(kScanColWarps * 32) sa_scan_cols_kernel(const SaNode *__restrict__ nodes,
                                                                          const int2 *__restrict__ groups,
                                                                          int32_t *__restrict__ tab) {
    const int2 gr = groups[blockIdx.x];   // (node, first column)
    const SaNode nd = nodes[gr.x];
    const int W = nd.G + 1, NG = nd.NR + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int h = gr.y + lane;
    const bool act = h < W;
    int32_t *col = tab + nd.tab_off + h;   // entry (g, h) at col[g W]
    const int per = (NG + kScanColWarps - 1) / kScanColWarps, g0 = min(NG, warp * per), g1 = min(NG, g0 + per);
    __shared__ int32_t part[kScanColWarps][32];
    int sum = 0;
    if (act)
#pragma unroll 4
        for (int g = g0; g < g1; ++g) sum += col[(int64_t) g * W];
    part[warp][lane] = sum;
    __syncthreads();
    int run = 0;
    for (int w = 0; w < warp; ++w) run += part[w][lane];
    if (act)
        for (int g = g0; g < g1; ++g) {
            const int v = col[(int64_t) g * W];
            col[(int64_t) g * W] = run;
            run += v;
        }
}

__device__ __forceinline__ int hbm_delta_corner(const SaNode &nd, const int32_t *tab, const int32_t *vec, int g, int h) {
    // delta(g Sr, h Sc) = #{hi: row < g Sr, col < h Sc} - #{lo: row < g Sr, col < h Sc}
    //                    + #{lo: row < g Sr} + #{lo: col < h Sc} - #lo       (tab holds the signed prefix)
    const int W = nd.G + 1;
    return tab[nd.tab_off + (int64_t) g * W + h] + vec[nd.vec_off + g] + vec[nd.vec_off + nd.NR + 1 + h] - nd.h;
}

template <int U = 1>
__device__ __forceinline__ int hbm_row_count(const int32_t *xs, int64_t off, int r0, int r1, int c, int lane) {
    return ballot_count<U>(r0, r1, lane, [&](int r) {
        const int v = xs[off + r];
        const int x = v & kValMask;
        return (v & kHiBit) ? (x < c) : (x >= c);
    });
}

template <int U = 1>
__device__ __forceinline__ int hbm_col_search(const int32_t *ys, int64_t off, int k, int from, int need, int R, int lane) {
    return ballot_search<U>(from, k, need, k + 1, lane, [&](int g) {
        const int w = ys[off + g];
        const int y = w & kValMask;
        return (w & kHiBit) ? (y < R) : (y >= R);
    });
}

// c* at the band boundaries R = b kBand that are multiples of Sc (one warp each): the table locates the
// column block, a ballot scan of at most Sc columns finds the column.
__global__ void __launch_bounds__(256) sa_coarse_kernel(const SaNode *__restrict__ nodes, const int2 *__restrict__ tasks,
                                                        int ntasks, const int32_t *__restrict__ tab,
                                                        const int32_t *__restrict__ vec, const int32_t *__restrict__ ys,
                                                        int32_t *__restrict__ cst) {
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (t >= ntasks) return;
    const int2 tk = tasks[t];   // (node, band)
    const SaNode nd = nodes[tk.x];
    const int R = tk.y * kBand, g = R / nd.Sr;
    // first h with delta(R, min(h Sc, k)) >= 0
    const int l = warp_first_true(0, nd.G + 1, lane, [&](int h) { return hbm_delta_corner(nd, tab, vec, g, h) >= 0; });
    int c;
    if (l == 0) c = 0;
    else if (l > nd.G) c = nd.k + 1;
    else {
        const int need = -hbm_delta_corner(nd, tab, vec, g, l - 1);
        c = hbm_col_search<4>(ys, nd.off, nd.k, (l - 1) * nd.Sc, need, R, lane);
    }
    if (lane == 0) cst[nd.cst_off + tk.y] = c;
}

// c* at the band boundaries that are not multiples of Sc (only when Sc > kBand), from the coarse boundary
// below: delta(R, c) = delta(Rb, c) - #{rows in [R, Rb) whose point raises delta at c}.
__global__ void __launch_bounds__(256) sa_fine_kernel(const SaNode *__restrict__ nodes, const int2 *__restrict__ tasks,
                                                      int ntasks, const int32_t *__restrict__ xs,
                                                      const int32_t *__restrict__ ys, int32_t *__restrict__ cst) {
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (t >= ntasks) return;
    const int2 tk = tasks[t];   // (node, band)
    const SaNode nd = nodes[tk.x];
    const int R = tk.y * kBand;
    const int Rb = min((R / nd.Sr + 1) * nd.Sr, nd.k);
    const int cb = Rb >= nd.k ? 0 : cst[nd.cst_off + Rb / kBand];
    int c = nd.k + 1;
    if (cb <= nd.k) {
        const int need = hbm_row_count<4>(xs, nd.off, R, Rb, cb, lane);
        c = hbm_col_search<4>(ys, nd.off, nd.k, cb, need, R, lane);
    }
    if (lane == 0) cst[nd.cst_off + tk.y] = c;
}

// ---- band kernel: the ant passage over kBand rows of one node, in shared memory ----

struct BandShared {
    int32_t x[kBand];                  // the band's rows: col | hi bit, replaced by the product
    int32_t y[kBandYCap];              // columns [clo, clo + ny): row | hi bit (when they fit)
    int32_t cst[kBandThreads + 1];     // c* at band rows kBandWalk * j; entry nwalk: the band's bottom
    int32_t queue[kBandThreads];       // walks left to whole warps
    int32_t subcnt[kBandThreads / 32]; // rows of each sub-band raising delta at the band's bottom c*
    int nq;
};

// Column points of the node: from shared memory when the band's column range was staged, else from global memory
// with, in shared memory, a table over blocks of B columns of [clo, cend) (built by build_wide_tables):
//   stat[b]  columns of block b whose point raises delta for every row of the band (hi points of rows < R0, lo
//            points of rows >= R1);
//   bend[b]  end in dyn of block b's points of the band's own rows [R0, R1) (block b: dyn[bend[b-1] .. bend[b]));
//   dyn[e]   such a point: its row offset i (row R0 + i) and hi bit (bit 15), which raises delta in row R iff
//            hi ? R0 + i < R : R0 + i >= R.
// A block's raising count for row R is then stat[b] plus a scan of its few own-row points: a search skips whole
// blocks and reads columns from global memory only in the block where it ends.
struct YView {
    const int32_t *s;   // shared copy of columns [clo, clo + ny)
    const int32_t *g;   // the node's columns in global memory
    int clo;
    bool in_smem;
    const uint16_t *stat;
    const int32_t *bend;
    const uint16_t *dyn;
    int B, nblk, R0;
    __device__ __forceinline__ int operator()(int c) const { return in_smem ? s[c - clo] : __ldg(g + c); }
    // raising columns of full block b for row R
    __device__ __forceinline__ int block_count(int b, int R) const {
        int cnt = stat[b];
        for (int e = b ? bend[b - 1] : 0, ee = bend[b]; e < ee; ++e) {
            const int d = dyn[e];
            const int r = R0 + (d & 0x0fff);
            cnt += (d & 0x8000) ? (r < R) : (r >= R);
        }
        return cnt;
    }
};

// warp-wide: rows i in [i0, i1) of the band whose point raises delta when moving up past it at column c
template <int U = 1>
__device__ __forceinline__ int band_row_count(const int32_t *X, int i0, int i1, int c, int lane) {
    return ballot_count<U>(i0, i1, lane, [&](int i) {
        const int v = X[i];
        const int x = v & kValMask;
        return (v & kHiBit) ? (x < c) : (x >= c);
    });
}

// warp-wide: as ballot_search, but in rounds that grow: the first 32 candidates alone, the next 128 together, then
// 1024 per round.  Most searches end within a few columns, while a long one (a band whose column range spans a
// large part of the node, as in the glue of the braids of two similar strings, read from global memory) then takes
// one load latency per 1024 columns instead of per 32.
template <typename Pred>
__device__ __forceinline__ int ballot_search_grow(int from, int end, int need, int none, int lane, Pred pred) {
    if (need <= 0) return from;
    const int g = from + lane;
    const unsigned m = __ballot_sync(kFull, g < end && pred(g));
    const int cnt = __popc(m);
    if (need <= cnt) return from + (int) __fns(m, 0, need) + 1;
    need -= cnt;
    const int mid = min(end, from + 32 + 128);
    int t = 0;   // raising candidates in [from + 32, mid)
    {
        bool q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int h = from + 32 + 32 * u + lane;
            q[u] = h < mid && pred(h);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned mu = __ballot_sync(kFull, q[u]);
            const int c = __popc(mu);
            if (t + c >= need) return from + 32 + 32 * u + (int) __fns(mu, 0, need - t) + 1;
            t += c;
        }
    }
    return ballot_search<32>(mid, end, need - t, none, lane, pred);
}

// warp-wide, columns in global memory (a band whose column range was too wide to stage): one past the need-th
// column g in [from, end) whose point raises delta in row R, `none` if there are fewer (need then reduced by the
// raising columns of the range).  Rounds of 512 columns, each
// lane loading its 16 columns unconditionally (indices clamped into the range) before testing any, so that a round
// costs one load latency: a search across the step of a nearly step-shaped demarcation line spans most of the node.
__device__ __forceinline__ int global_col_search(const int32_t *__restrict__ ycol, int from, int end, int &need, int R,
                                                 int none, int lane) {
    constexpr int U = 16;
    for (int g0 = from; g0 < end; g0 += 32 * U) {
        int v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = __ldg(ycol + min(g0 + 32 * u + lane, end - 1));
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int y = v[u] & kValMask;
            const bool q = g0 + 32 * u + lane < end && ((v[u] & kHiBit) ? (y < R) : (y >= R));
            const unsigned m = __ballot_sync(kFull, q);
            const int cnt = __popc(m);
            if (need <= cnt) return g0 + 32 * u + (int) __fns(m, 0, need) + 1;
            need -= cnt;
        }
    }
    return none;
}

// warp-wide, columns in global memory with the block table of Y: as global_col_search.  The head up to the first
// block boundary and the block where the search ends are scanned in global memory; the blocks between are
// counted from the table, 32 per round (lane = block, a prefix sum over the lanes).
__device__ __forceinline__ int wide_col_search(const YView &Y, int from, int cend, int need, int R, int none,
                                               int lane) {
    const int B = Y.B;
    int b = (from - Y.clo + B - 1) / B;                    // first full block at or after `from`
    const int head_end = min(cend, Y.clo + b * B);
    if (from < head_end) {   // (on `none`, need has been reduced by the head's raising columns)
        const int c = global_col_search(Y.g, from, head_end, need, R, none, lane);
        if (c != none) return c;
    }
    const int bfull = min(Y.nblk, (cend - Y.clo) / B);   // blocks entirely below cend
    for (; b < bfull; b += 32) {
        const int bl = b + lane;
        const int cnt = bl < bfull ? Y.block_count(bl, R) : 0;
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        const int tot = __shfl_sync(kFull, incl, 31);
        if (tot < need) {
            need -= tot;
            continue;
        }
        const int j = __ffs(__ballot_sync(kFull, incl >= need)) - 1;
        const int before = __shfl_sync(kFull, incl - cnt, j);
        const int g0 = Y.clo + (b + j) * B;
        need -= before;
        return global_col_search(Y.g, g0, g0 + B, need, R, none, lane);
    }
    const int tail = max(head_end, Y.clo + bfull * B);
    return tail < cend ? global_col_search(Y.g, tail, cend, need, R, none, lane) : none;
}

// warp-wide: one past the need-th column g in [from, cend) whose point raises delta in row R; k + 1 if none
// (U = 0: the growing search above on staged columns; columns left in global memory take the block table)
template <int U = 0>
__device__ __forceinline__ int band_col_search(const YView &Y, int k, int from, int cend, int need, int R, int lane) {
    if (need <= 0) return from;
    if (!Y.in_smem) return wide_col_search(Y, from, cend, need, R, k + 1, lane);
    auto pred = [&](int g) {
        const int w = Y.s[g - Y.clo];
        const int y = w & kValMask;
        return (w & kHiBit) ? (y < R) : (y >= R);
    };
    if constexpr (U == 0) return ballot_search_grow(from, cend, need, k + 1, lane, pred);
    else return ballot_search<U>(from, cend, need, k + 1, lane, pred);
}

// one thread: band rows [i0, i1) walked up from c = c*(R0 + i1)
__device__ __forceinline__ void band_thread_walk(int32_t *X, const YView &Y, int k, int R0, int i0, int i1, int c,
                                                 int cend) {
    for (int i = i1 - 1; i >= i0; --i) {
        const int v = X[i];
        const int xr = v & kValMask;
        const bool hi = v & kHiBit;
        if (hi ? (xr < c) : (xr >= c)) {
            const int r = R0 + i;
            int g = c;
            for (; g < cend; ++g) {
                const int w = Y(g);
                const int yr = w & kValMask;
                if ((w & kHiBit) ? (yr < r) : (yr >= r)) break;
            }
            c = g < cend ? g + 1 : k + 1;
        }
        const bool good = c >= 1 && c <= k && (hi ? (xr < c) : (xr >= c));
        X[i] = good ? c - 1 : xr;
    }
}

// one warp: the same walk for a walk whose columns span is long; rows without a jump are settled 32 at a
// time by a ballot, every jump is a ballot scan of the columns
__device__ __forceinline__ void band_warp_walk(int32_t *X, const YView &Y, int k, int R0, int i0, int i1, int c,
                                               int cend, int lane) {
    int ib = i1;   // rows [ib, i1) are done
    while (ib > i0) {
        const int i = ib - 1 - lane;
        int v = 0;
        bool ind = false;
        if (i >= i0) {
            v = X[i];
            const int x = v & kValMask;
            ind = (v & kHiBit) ? (x < c) : (x >= c);
        }
        const unsigned m = __ballot_sync(kFull, ind);
        const int j = m ? __ffs(m) - 1 : 32;   // lanes below j keep their point
        if (lane < j && i >= i0) X[i] = v & kValMask;
        if (j == 32) {
            ib -= 32;
            continue;
        }
        const int ij = ib - 1 - j;
        const int vj = __shfl_sync(kFull, v, j);
        c = band_col_search(Y, k, c, cend, 1, R0 + ij, lane);
        const int xr = vj & kValMask;
        const bool good = c >= 1 && c <= k && ((vj & kHiBit) ? (xr < c) : (xr >= c));
        if (lane == 0) X[ij] = good ? c - 1 : xr;
        ib = ij;
    }
    __syncwarp();
}

// The block table of a band whose columns [clo, clo + nblk B) stay in global memory (the whole CTA; wbend zeroed
// and S.x loaded before): per block its static raising count (one warp per run of blocks, 8 loads in flight per
// lane), then the band's own points bucketed by block (counts, an exclusive scan over the blocks, a scatter that
// leaves wbend[b] = end of bucket b).  `tmp`: kBandThreads ints of scratch.
__device__ __forceinline__ void build_wide_tables(const int32_t *__restrict__ ycol, const int32_t *X, int nr, int R0,
                                                  int clo, int B, int nblk, uint16_t *wstat, int32_t *wbend,
                                                  uint16_t *wdyn, int32_t *tmp, int tid) {
    constexpr int V = 8;
    constexpr int nwarps = kBandThreads / 32;
    const int lane = tid & 31, warp = tid >> 5;
    const int R1 = R0 + nr;
    {
        const int bw0 = (int) ((long long) nblk * warp / nwarps), bw1 = (int) ((long long) nblk * (warp + 1) / nwarps);
        const int start = clo + bw0 * B, end = clo + bw1 * B;
        int cur = bw0, acc = 0;
        for (int g0 = start; g0 < end; g0 += 32 * V) {
            int v[V];
#pragma unroll
            for (int u = 0; u < V; ++u) v[u] = __ldg(ycol + min(g0 + 32 * u + lane, end - 1));
#pragma unroll
            for (int u = 0; u < V; ++u) {
                const int chunk = g0 + 32 * u;
                if (chunk < end) {   // warp-uniform
                    const int y = v[u] & kValMask;
                    const bool st = (v[u] & kHiBit) ? (y < R0) : (y >= R1);
                    const int cnt = __popc(__ballot_sync(kFull, st));
                    const int blk = (chunk - clo) / B;
                    if (blk != cur) {
                        if (lane == 0) wstat[cur] = (uint16_t) acc;
                        acc = 0;
                        cur = blk;
                    }
                    acc += cnt;
                }
            }
        }
        if (lane == 0 && bw0 < bw1) wstat[cur] = (uint16_t) acc;
    }
    const int cend = clo + nblk * B;
    for (int i = tid; i < nr; i += kBandThreads) {
        const int c = X[i] & kValMask;
        if (c >= clo && c < cend) atomicAdd(&wbend[(c - clo) / B], 1);
    }
    __syncthreads();
    // exclusive scan of the bucket counts: a segment per thread, then the segment sums across the CTA
    const int seg = (nblk + kBandThreads - 1) / kBandThreads;
    const int s0 = min(nblk, tid * seg), s1 = min(nblk, s0 + seg);
    int sum = 0;
    for (int b = s0; b < s1; ++b) sum += wbend[b];
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) tmp[warp] = incl;
    __syncthreads();
    int base = incl - sum;
    for (int w = 0; w < warp; ++w) base += tmp[w];
    for (int b = s0; b < s1; ++b) {
        const int c = wbend[b];
        wbend[b] = base;
        base += c;
    }
    __syncthreads();
    for (int i = tid; i < nr; i += kBandThreads) {
        const int v = X[i];
        const int c = v & kValMask;
        if (c >= clo && c < cend) {
            const int pos = atomicAdd(&wbend[(c - clo) / B], 1);
            wdyn[pos] = (uint16_t) (i | ((v & kHiBit) ? 0x8000 : 0));
        }
    }
}

// One CTA per band of kBand rows of a node: c* at every kBandSub rows (scans from the band's bottom), then
// at every kBandWalk rows (each warp bottom-up through its sub-band), then walks of kBandWalk rows.
__global__ void __launch_bounds__(kBandThreads, 3) sa_band_kernel(const SaNode *__restrict__ nodes,
                                                               const int2 *__restrict__ tasks,
                                                               const int32_t *__restrict__ xs,
                                                               const int32_t *__restrict__ ys,
                                                               const int32_t *__restrict__ cst,
                                                               int32_t *__restrict__ RESout) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BandShared &S = *reinterpret_cast<BandShared *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int nwarps = kBandThreads / 32;
    constexpr int wsub = kBandSub / kBandWalk;   // walks per sub-band
    const int2 tk = tasks[blockIdx.x];   // (node, band)
    const SaNode nd = nodes[tk.x];
    const int k = nd.k, R0 = tk.y * kBand, R1 = min(R0 + kBand, k), nr = R1 - R0;
    const int ctop = cst[nd.cst_off + tk.y];
    const int cbot = R1 >= k ? 0 : cst[nd.cst_off + tk.y + 1];
    // columns the band can read: [clo, cend) (c* only grows walking up, and stops at ctop)
    const int cend = min(ctop, k);
    const int clo = min(cbot, cend);
    const int ny = cend - clo;
    const bool ysm = ny <= kBandYCap;
    const int nwalk = (nr + kBandWalk - 1) / kBandWalk;
    // staging, eight loads in flight per thread
    for (int i0 = 0; i0 < nr; i0 += 8 * kBandThreads) {
        int v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + tid + kBandThreads * u;
            v[u] = i < nr ? xs[nd.off + R0 + i] : 0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (i0 + tid + kBandThreads * u < nr) S.x[i0 + tid + kBandThreads * u] = v[u];
    }
    if (ysm)
        for (int i0 = 0; i0 < ny; i0 += 8 * kBandThreads) {
            int v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int i = i0 + tid + kBandThreads * u;
                v[u] = i < ny ? ys[nd.off + clo + i] : 0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (i0 + tid + kBandThreads * u < ny) S.y[i0 + tid + kBandThreads * u] = v[u];
        }
    if (tid == 0) {
        S.cst[0] = ctop;
        S.cst[nwalk] = cbot;
        S.nq = 0;
    }
    // columns left in global memory: the block table (YView) in the space of the staging area
    int B = 0, nblk = 0;
    uint16_t *wstat = reinterpret_cast<uint16_t *>(S.y);
    int32_t *wbend = nullptr;
    uint16_t *wdyn = nullptr;
    if (!ysm) {
        B = 32 * ((ny + 32 * kWideMaxBlocks - 1) / (32 * kWideMaxBlocks));
        nblk = ny / B;
        wbend = reinterpret_cast<int32_t *>(wstat + ((nblk + 1) & ~1));
        wdyn = reinterpret_cast<uint16_t *>(wbend + nblk);
        for (int b = tid; b < nblk; b += kBandThreads) wbend[b] = 0;
    }
    __syncthreads();
    if (!ysm) {
        build_wide_tables(ys + nd.off, S.x, nr, R0, clo, B, nblk, wstat, wbend, wdyn, S.queue, tid);
        __syncthreads();
    }
    const YView Y{S.y, ys + nd.off, clo, ysm, wstat, wbend, wdyn, B, nblk, R0};
    // c* at the sub-band tops (warp w >= 1: row R0 + w kBandSub).  The rows between a top and the band's bottom
    // that raise delta at cbot are counted once per sub-band (each warp its own), and summed over the warps below.
    if (cbot <= k && warp * kBandSub < nr) {
        const int i0 = warp * kBandSub, i1 = min(i0 + kBandSub, nr);
        const int cnt = band_row_count<4>(S.x, i0, i1, cbot, lane);
        if (lane == 0) S.subcnt[warp] = cnt;
    }
    __syncthreads();
    if (warp >= 1 && warp * kBandSub < nr) {
        const int i = warp * kBandSub;
        int c = k + 1;
        if (cbot <= k) {
            int need = 0;
            for (int w = warp; w < nwarps && w * kBandSub < nr; ++w) need += S.subcnt[w];
            c = band_col_search<4>(Y, k, cbot, cend, need, R0 + i, lane);
        }
        if (lane == 0) S.cst[warp * wsub] = c;
    }
    __syncthreads();
    // c* at every walk top inside each sub-band, bottom-up from the boundary below it
    if (warp * kBandSub < nr) {
        const int jtop = warp * wsub, jbot = min((warp + 1) * wsub, nwalk);
        int cb = S.cst[jbot];
        for (int j = jbot - 1; j > jtop; --j) {
            const int i = j * kBandWalk, ie = min(i + kBandWalk, nr);
            int c = k + 1;
            if (cb <= k) {
                const int need = band_row_count(S.x, i, ie, cb, lane);
                c = band_col_search(Y, k, cb, cend, need, R0 + i, lane);
            }
            if (lane == 0) S.cst[j] = c;
            cb = c;
        }
    }
    __syncthreads();
    // walks: short column spans by one thread each, long ones queued for whole warps
    if (tid < nwalk) {
        const int i0 = tid * kBandWalk, i1 = min(i0 + kBandWalk, nr);
        const int c0 = S.cst[tid + 1], ce = S.cst[tid];
        // (with the columns in global memory every walk goes to a warp: a thread's column scan would be a chain of
        // dependent loads)
        if (ysm && min(ce, k) - min(c0, k) <= kWalkSpanMax) band_thread_walk(S.x, Y, k, R0, i0, i1, c0, cend);
        else S.queue[atomicAdd(&S.nq, 1)] = tid;
    }
    __syncthreads();
    for (int q = warp; q < S.nq; q += nwarps) {
        const int t = S.queue[q];
        const int i0 = t * kBandWalk, i1 = min(i0 + kBandWalk, nr);
        band_warp_walk(S.x, Y, k, R0, i0, i1, S.cst[t + 1], cend, lane);
    }
    __syncthreads();
    for (int i = tid; i < nr; i += kBandThreads) RESout[nd.off + R0 + i] = S.x[i];
}

// Nodes without a sibling at this level carry their lists and product over unchanged.
__global__ void sa_copy_kernel(const int64_t *__restrict__ ranges, int nranges, const int32_t *__restrict__ a0,
                               const int32_t *__restrict__ b0, const int32_t *__restrict__ c0, int32_t *__restrict__ a1,
                               int32_t *__restrict__ b1, int32_t *__restrict__ c1) {
    for (int r = blockIdx.y; r < nranges; r += gridDim.y) {
        const int64_t off = ranges[2 * r], len = ranges[2 * r + 1];
        for (int64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t) gridDim.x * blockDim.x) {
            a1[off + i] = a0[off + i];
            b1[off + i] = b0[off + i];
            c1[off + i] = c0[off + i];
        }
    }
}

// P^-1 of every problem: Pinv[off + P(r)] = r.
__global__ void sa_pinv_kernel(const SaNode *__restrict__ probs, const SaTile *__restrict__ tiles,
                               const int32_t *__restrict__ P, int32_t *__restrict__ Pinv, int *err) {
    const SaTile tl = tiles[blockIdx.x];
    const SaNode pr = probs[tl.node];
    const int e0 = tl.t * kMT, e1 = min(e0 + kMT, pr.k);
    for (int r = e0 + threadIdx.x; r < e1; r += blockDim.x) {
        const int c = P[pr.off + r];
        if (c < 0 || c >= pr.k) {
            raise_error(err, kDevErrBadState);
            continue;
        }
        Pinv[pr.off + c] = r;
    }
}


struct SaLevel {
    int64_t size;                 // children size at this level (node span = 2 size)
    int nnodes, ntiles, nl0, nl1, nct, nft, nwt, ncopies;
    int64_t o_nodes, o_tiles, o_l0, o_l1, o_ct, o_ft, o_wt, o_copies;   // offsets into the plan arrays
    int64_t tab_tot, vec_tot, cst_tot;
    std::vector<int> finished;    // problems whose root is produced at this level
};


}  // namespace

struct SaPlan {
    std::vector<int64_t> off;
    std::vector<int> n;
    int np = 0;
    int64_t total = 0;
    int maxn = 0;
    int nprobtiles = 0, nitems = 0;
    std::vector<int> small;   // problems finished by the shared-memory kernel
    std::vector<SaLevel> levels;
    // device
    SaNode *d_probs = nullptr;
    SaTile *d_probtiles = nullptr;
    SaBlockItem *d_items = nullptr;
    SaNode *d_nodes = nullptr;
    SaTile *d_tiles = nullptr;
    int2 *d_tasks = nullptr;
    int64_t *d_copies = nullptr;
    int2 *d_splits = nullptr;     // merge-path splits of the merge tiles of one level
    int max_tiles = 0;
    int32_t *pinv = nullptr, *pl[2] = {nullptr, nullptr}, *ql[2] = {nullptr, nullptr}, *res[2] = {nullptr, nullptr};
    int32_t *posP = nullptr, *posQ = nullptr, *xs = nullptr, *ys = nullptr, *tab = nullptr, *vec = nullptr,
            *cst = nullptr;
    int64_t tab_max = 0, vec_max = 0, cst_max = 0;
    int max_w = 0;                 // widest block table (G + 1) of any level
    cudaStream_t alloc_stream = nullptr;
    bool shared_scratch = false;   // per-element scratch owned by the caller
};

namespace {
template <typename T>
int plan_upload(T **dst, const std::vector<T> &v, cudaStream_t s) {
    SLCS_TRY(dalloc(reinterpret_cast<void **>(dst), sizeof(T) * std::max<size_t>(v.size(), 1), s));
    if (!v.empty()) SLCS_CUDA_TRY(cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
    return SLCS_OK;
}
}  // namespace

// Points a plan created with deferred shared scratch at the caller's buffers.
int sa_plan_bind(SaPlan *P, const SaScratch *sh) {
    if (sh->elems < std::max<int64_t>(P->total, 1) || sh->tab < P->tab_max || sh->vec < P->vec_max || sh->cst < P->cst_max)
        return fail(SLCS_ERR_INTERNAL, "steady-ant shared scratch too small");
    P->pinv = sh->b[0];
    P->pl[0] = sh->b[1];
    P->pl[1] = sh->b[2];
    P->ql[0] = sh->b[3];
    P->ql[1] = sh->b[4];
    P->res[0] = sh->b[5];
    P->res[1] = sh->b[6];
    P->posP = sh->b[7];
    P->posQ = sh->b[8];
    P->xs = sh->b[9];
    P->ys = sh->b[10];
    P->tab = sh->tabp;
    P->vec = sh->vecp;
    P->cst = sh->cstp;
    return SLCS_OK;
}

void sa_plan_destroy(SaPlan *P) {
    if (!P) return;
    cudaStream_t s = P->alloc_stream;
    void *ptrs[] = {P->d_probs, P->d_probtiles, P->d_items, P->d_nodes, P->d_tiles, P->d_tasks, P->d_copies,
                    P->d_splits};
    for (void *p : ptrs) dfree(p, s);
    if (!P->shared_scratch) {
        void *sp[] = {P->pinv, P->pl[0], P->pl[1], P->ql[0], P->ql[1], P->res[0], P->res[1], P->posP, P->posQ,
                      P->xs, P->ys, P->tab, P->vec, P->cst};
        for (void *p : sp) dfree(p, s);
    }
    delete P;
}

void sa_plan_set_stream(SaPlan *P, cudaStream_t s) {
    if (P) P->alloc_stream = s;
}

// Plans the batched unit-Monge products of problems i = 0..np-1, problem i occupying [off[i], off[i] + n[i])
// of concatenated row->col arrays.  All task lists and scratch are built and allocated here.
int sa_plan_create(const std::vector<int64_t> &off, const std::vector<int> &n, SaPlan **out, cudaStream_t s,
                   const SaScratch *shared, int cutoff) {
    // sub-problems of at most `cut` common indices finish in shared memory (a power of two <= kSaSB)
    int cut = cutoff > 0 ? cutoff : pick_sa_cutoff();
    {
        int c = 256;
        while (c * 2 <= cut && c < kSaSB) c <<= 1;
        cut = c;
    }
    *out = nullptr;
    auto P = new SaPlan();
    P->alloc_stream = s;
    P->off = off;
    P->n = n;
    P->np = (int) n.size();
    for (int i = 0; i < P->np; ++i) {
        P->total = std::max<int64_t>(P->total, off[i] + n[i]);
        P->maxn = std::max(P->maxn, n[i]);
    }
    auto bail = [&](int rc) {
        sa_plan_destroy(P);
        return rc;
    };
    std::vector<SaNode> probs(P->np);
    std::vector<SaTile> probtiles;
    std::vector<SaBlockItem> items;
    for (int i = 0; i < P->np; ++i) {
        if (n[i] > 0 && n[i] <= cut) P->small.push_back(i);
        probs[i] = SaNode{off[i], n[i], n[i], 0, 0, 0, 0, 0};
        for (int t = 0; (int64_t) t * kMT < n[i]; ++t) probtiles.push_back(SaTile{i, t});
        for (int b0 = 0; b0 < n[i]; b0 += cut) items.push_back(SaBlockItem{off[i] + b0, std::min(cut, n[i] - b0), 0});
    }
    P->nprobtiles = (int) probtiles.size();
    P->nitems = (int) items.size();
    std::vector<SaNode> nodes;
    std::vector<SaTile> tiles;
    std::vector<int2> tasks;
    std::vector<int64_t> copies;
    for (int64_t size = cut; size < P->maxn; size <<= 1) {
        const int64_t span = size << 1;
        SaLevel L{};
        L.size = size;
        L.o_nodes = (int64_t) nodes.size();
        L.o_copies = (int64_t) copies.size();
        const size_t first_node = nodes.size();
        for (int i = 0; i < P->np; ++i) {
            if (n[i] <= size) continue;
            if (n[i] <= span) L.finished.push_back(i);
            for (int64_t a = 0; a < n[i]; a += span) {
                const int k = (int) std::min<int64_t>(span, n[i] - a);
                const int h = (int) std::min<int64_t>(size, k);
                if (h == k) {
                    copies.push_back(off[i] + a);
                    copies.push_back(k);
                    continue;
                }
                int Sc = 256;
                while ((int64_t) Sc * Sc < k) Sc <<= 1;
                while (Sc < kBand && k / Sc > 1024) Sc <<= 1;   // a (G+1)^2 table of at most ~1024^2 entries
                const int G = (k + Sc - 1) / Sc;
                const int Sr = std::max(Sc, kBand), NR = (k + Sr - 1) / Sr;
                nodes.push_back(SaNode{off[i] + a, k, h, Sc, G, Sr, NR, L.tab_tot, L.vec_tot, L.cst_tot});
                L.tab_tot += (int64_t) (NR + 1) * (G + 1);
                L.vec_tot += (int64_t) (NR + 1) + (G + 1);
                L.cst_tot += (k + kBand - 1) / kBand + 1;
            }
        }
        L.nnodes = (int) (nodes.size() - first_node);
        L.ncopies = (int) ((copies.size() - L.o_copies) / 2);
        L.o_tiles = (int64_t) tiles.size();
        for (int j = 0; j < L.nnodes; ++j)
            for (int t = 0; (int64_t) t * kMT < nodes[first_node + j].k; ++t) tiles.push_back(SaTile{j, t});
        L.ntiles = (int) (tiles.size() - L.o_tiles);
        P->max_tiles = std::max(P->max_tiles, L.ntiles);
        L.o_l0 = (int64_t) tasks.size();
        for (int j = 0; j < L.nnodes; ++j) {
            for (int y = 0; y < nodes[first_node + j].NR + 1; ++y) tasks.push_back(make_int2(j, y));
            P->max_w = std::max(P->max_w, nodes[first_node + j].G + 1);
        }
        L.nl0 = (int) (tasks.size() - L.o_l0);
        L.o_l1 = (int64_t) tasks.size();
        for (int j = 0; j < L.nnodes; ++j)
            for (int y = 0; y < nodes[first_node + j].G + 1; y += 32) tasks.push_back(make_int2(j, y));
        L.nl1 = (int) (tasks.size() - L.o_l1);
        // band boundaries: from the table where they are multiples of Sc, else from the one below
        L.o_ct = (int64_t) tasks.size();
        for (int j = 0; j < L.nnodes; ++j) {
            const SaNode &nd = nodes[first_node + j];
            for (int b = 0; (int64_t) b * kBand < nd.k; ++b)
                if (((int64_t) b * kBand) % nd.Sr == 0) tasks.push_back(make_int2(j, b));
        }
        L.nct = (int) (tasks.size() - L.o_ct);
        L.o_ft = (int64_t) tasks.size();
        for (int j = 0; j < L.nnodes; ++j) {
            const SaNode &nd = nodes[first_node + j];
            for (int b = 0; (int64_t) b * kBand < nd.k; ++b)
                if (((int64_t) b * kBand) % nd.Sr != 0) tasks.push_back(make_int2(j, b));
        }
        L.nft = (int) (tasks.size() - L.o_ft);
        L.o_wt = (int64_t) tasks.size();
        for (int j = 0; j < L.nnodes; ++j)
            for (int b = 0; (int64_t) b * kBand < nodes[first_node + j].k; ++b) tasks.push_back(make_int2(j, b));
        L.nwt = (int) (tasks.size() - L.o_wt);
        if ((int64_t) P->max_w * (int64_t) sizeof(int32_t) > kRowHistSmemMax)
            return bail(fail(SLCS_ERR_ARG, "steady ant: product too large for the block-table histogram"));
        P->tab_max = std::max(P->tab_max, L.tab_tot);
        P->vec_max = std::max(P->vec_max, L.vec_tot);
        P->cst_max = std::max(P->cst_max, L.cst_tot);
        P->levels.push_back(std::move(L));
    }
    int rc;
    if ((rc = plan_upload(&P->d_probs, probs, s)) || (rc = plan_upload(&P->d_probtiles, probtiles, s)) ||
        (rc = plan_upload(&P->d_items, items, s)) || (rc = plan_upload(&P->d_nodes, nodes, s)) ||
        (rc = plan_upload(&P->d_tiles, tiles, s)) || (rc = plan_upload(&P->d_tasks, tasks, s)) ||
        (rc = plan_upload(&P->d_copies, copies, s)) ||
        (rc = dalloc(reinterpret_cast<void **>(&P->d_splits), sizeof(int2) * std::max(P->max_tiles, 1), s)))
        return bail(rc);
    const int64_t T = std::max<int64_t>(P->total, 1);
    if (shared) {
        P->shared_scratch = true;
        if (shared->elems >= 0 && (rc = sa_plan_bind(P, shared))) return bail(rc);
    } else {
        int32_t **bufs1[] = {&P->pinv, &P->pl[0], &P->ql[0], &P->res[0]};
        for (auto b : bufs1)
            if ((rc = dalloc(reinterpret_cast<void **>(b), sizeof(int32_t) * T, s))) return bail(rc);
        if (!P->levels.empty()) {
            int32_t **bufs2[] = {&P->pl[1], &P->ql[1], &P->res[1], &P->posP, &P->posQ, &P->xs, &P->ys};
            for (auto b : bufs2)
                if ((rc = dalloc(reinterpret_cast<void **>(b), sizeof(int32_t) * T, s))) return bail(rc);
            if ((rc = dalloc(reinterpret_cast<void **>(&P->tab), sizeof(int32_t) * std::max<int64_t>(P->tab_max, 1), s)) ||
                (rc = dalloc(reinterpret_cast<void **>(&P->vec), sizeof(int32_t) * std::max<int64_t>(P->vec_max, 1), s)) ||
                (rc = dalloc(reinterpret_cast<void **>(&P->cst), sizeof(int32_t) * std::max<int64_t>(P->cst_max, 1), s)))
                return bail(rc);
        }
    }
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(sa_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int) sizeof(SaShared));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(sa_band_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sizeof(BandShared));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(sa_rowhist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowHistSmemMax);
        if (e != cudaSuccess) return bail(fail(SLCS_ERR_CUDA, "cudaFuncSetAttribute(steady-ant kernels) failed"));
        attr_set = true;
    }
    *out = P;
    return SLCS_OK;
}

// Runs a plan: kernels only (no host synchronisation, no allocation), so the sequence can be captured.
// Runs a plan: kernels only (no host synchronisation, no allocation), so the sequence can be captured.
// Permutation mode (d_leafP == nullptr): d_P, d_Q are row->col permutations, d_R receives the product.
// Leaf mode: d_leafP[j] / d_Q[j] give, for common index j of each problem, the (distinct, arbitrary) id of
// P's row with column j and of Q's column with row j; the roots' sorted id lists go to d_PLout / d_QLout and
// the product in root-local coordinates (rank of row id -> rank of column id) to d_R.
int sa_plan_run_ex(SaPlan *P, const int32_t *d_P, const int32_t *d_leafP, const int32_t *d_Q, int32_t *d_R,
                   int32_t *d_PLout, int32_t *d_QLout, int *d_err, cudaStream_t s) {
    NvtxRange nv("slcs: steady ant");
    if (P->total == 0) return SLCS_OK;
    const int32_t *leafP = d_leafP;
    if (!leafP) {
        if (P->nprobtiles) sa_pinv_kernel<<<P->nprobtiles, 256, 0, s>>>(P->d_probs, P->d_probtiles, d_P, P->pinv, d_err);
        leafP = P->pinv;
    }
    if (P->nitems)
        sa_block_kernel<<<P->nitems, kSaThreads, sizeof(SaShared), s>>>(leafP, d_Q, P->d_items, P->pl[0], P->ql[0],
                                                                        P->res[0], d_err);
    SLCS_CUDA_TRY(cudaGetLastError());
    auto emit_roots = [&](const std::vector<int> &probs, int buf) -> int {
        // consecutive problems are copied as one range
        for (size_t x = 0; x < probs.size();) {
            size_t y = x + 1;
            while (y < probs.size() && probs[y] == probs[y - 1] + 1 && P->off[probs[y]] == P->off[probs[y - 1]] + P->n[probs[y - 1]]) ++y;
            const int64_t o = P->off[probs[x]];
            const int64_t len = P->off[probs[y - 1]] + P->n[probs[y - 1]] - o;
            SLCS_CUDA_TRY(cudaMemcpyAsync(d_R + o, P->res[buf] + o, sizeof(int32_t) * len, cudaMemcpyDeviceToDevice, s));
            if (d_PLout)
                SLCS_CUDA_TRY(cudaMemcpyAsync(d_PLout + o, P->pl[buf] + o, sizeof(int32_t) * len, cudaMemcpyDeviceToDevice, s));
            if (d_QLout)
                SLCS_CUDA_TRY(cudaMemcpyAsync(d_QLout + o, P->ql[buf] + o, sizeof(int32_t) * len, cudaMemcpyDeviceToDevice, s));
            x = y;
        }
        return SLCS_OK;
    };
    SLCS_TRY(emit_roots(P->small, 0));
    int cur = 0;
    for (const SaLevel &L : P->levels) {
        const int nxt = cur ^ 1;
        const SaNode *nodes = P->d_nodes + L.o_nodes;
        if (L.nnodes) {
            const SaTile *tiles = P->d_tiles + L.o_tiles;
            sa_split_kernel<<<(2 * L.ntiles + 7) / 8, 256, 0, s>>>(nodes, tiles, L.ntiles, P->pl[cur], P->ql[cur],
                                                                  P->d_splits);
            sa_merge_kernel<<<dim3((unsigned) L.ntiles, 2), 256, 0, s>>>(nodes, tiles, P->d_splits, P->pl[cur], P->pl[nxt],
                                                                         P->posP, P->ql[cur], P->ql[nxt], P->posQ);
            sa_map_kernel<<<L.ntiles, 256, 0, s>>>(nodes, tiles, P->posP, P->posQ, P->res[cur], P->xs, P->ys, d_err);
            sa_rowhist_kernel<<<L.nl0, 256, sizeof(int32_t) * P->max_w, s>>>(nodes, P->d_tasks + L.o_l0, P->xs, P->posP,
                                                                             P->posQ, P->tab, P->vec);
            sa_scan_cols_kernel<<<L.nl1, kScanColWarps * 32, 0, s>>>(nodes, P->d_tasks + L.o_l1, P->tab);
            if (L.nct)
                sa_coarse_kernel<<<(L.nct + 7) / 8, 256, 0, s>>>(nodes, P->d_tasks + L.o_ct, L.nct, P->tab, P->vec,
                                                                 P->ys, P->cst);
            if (L.nft)
                sa_fine_kernel<<<(L.nft + 7) / 8, 256, 0, s>>>(nodes, P->d_tasks + L.o_ft, L.nft, P->xs, P->ys, P->cst);
            sa_band_kernel<<<L.nwt, kBandThreads, sizeof(BandShared), s>>>(nodes, P->d_tasks + L.o_wt, P->xs, P->ys,
                                                                           P->cst, P->res[nxt]);
            SLCS_CUDA_TRY(cudaGetLastError());
        }
        if (L.ncopies) {
            dim3 grid(64, (unsigned) std::min(L.ncopies, 65535));
            sa_copy_kernel<<<grid, 256, 0, s>>>(P->d_copies + L.o_copies, L.ncopies, P->pl[cur], P->ql[cur],
                                                P->res[cur], P->pl[nxt], P->ql[nxt], P->res[nxt]);
            SLCS_CUDA_TRY(cudaGetLastError());
        }
        SLCS_TRY(emit_roots(L.finished, nxt));
        cur = nxt;
    }
    return SLCS_OK;
}

int sa_plan_run(SaPlan *P, const int32_t *d_P, const int32_t *d_Q, int32_t *d_R, int *d_err, cudaStream_t s) {
    return sa_plan_run_ex(P, d_P, nullptr, d_Q, d_R, nullptr, nullptr, d_err, s);
}

int sa_plan_launches(const SaPlan *P) {
    int c = (P->nprobtiles ? 1 : 0) + (P->nitems ? 1 : 0);
    for (const SaLevel &L : P->levels) c += (L.nnodes ? 6 + (L.nct ? 1 : 0) + (L.nft ? 1 : 0) : 0) + (L.ncopies ? 1 : 0);
    return c;
}

int64_t sa_plan_total(const SaPlan *P) { return P->total; }

void sa_plan_needs(const SaPlan *P, int64_t *elems, int64_t *tab, int64_t *vec, int64_t *cst) {
    *elems = std::max<int64_t>(P->total, 1);
    *tab = P->tab_max;
    *vec = P->vec_max;
    *cst = P->cst_max;
}

int steady_ant_batch_dev(const int32_t *d_P, const int32_t *d_Q, const std::vector<int64_t> &off,
                         const std::vector<int> &n, int32_t *d_R, int *d_err, cudaStream_t s, int cutoff) {
    SaPlan *P = nullptr;
    SLCS_TRY(sa_plan_create(off, n, &P, s, nullptr, cutoff));
    int rc = sa_plan_run(P, d_P, d_Q, d_R, d_err, s);
    sa_plan_destroy(P);
    return rc;
}

int steady_ant_max_small() { return kSaSB; }

}  // namespace slcs

using namespace slcs;

extern "C" {

int slcs_steady_ant_dev(const int32_t *d_p, const int32_t *d_q, int n, int32_t *d_r, const slcs_opts *opts,
                        void *stream) {
    if (n < 0) return fail(SLCS_ERR_ARG, "negative size");
    if (n > 0 && (!d_p || !d_q || !d_r)) return fail(SLCS_ERR_ARG, "NULL buffer");
    if (n >= (1 << 30)) return fail(SLCS_ERR_TOO_LARGE, "n must be below 2^30");
    Engine *E;
    SLCS_TRY(engine(&E));
    if (n == 0) return SLCS_OK;
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    DevBuf<int> err;
    SLCS_TRY(err.alloc(1, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    SLCS_TRY(steady_ant_batch_dev(d_p, d_q, std::vector<int64_t>{0}, std::vector<int>{n}, d_r, err.p, s,
                                  opts ? opts->sa_cutoff : 0));
    return check_dev_err(err.p, s);
}

struct slcs_sa_plan {
    SaPlan *plan = nullptr;
    int *d_err = nullptr;
    int device = 0;
    int n = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const void *gp = nullptr, *gq = nullptr, *gr = nullptr;
};

int slcs_sa_plan_create(int n, slcs_sa_plan **out) {
    if (!out || n < 0 || n >= (1 << 30)) return fail(SLCS_ERR_ARG, "bad plan arguments");
    *out = nullptr;
    Engine *E;
    SLCS_TRY(engine(&E));
    auto h = new slcs_sa_plan();
    h->device = E->device;
    h->n = n;
    int rc = sa_plan_create(std::vector<int64_t>{0}, std::vector<int>{n}, &h->plan, E->stream, nullptr);
    if (rc == SLCS_OK) rc = dalloc(reinterpret_cast<void **>(&h->d_err), sizeof(int), E->stream);
    if (rc == SLCS_OK && cudaMemsetAsync(h->d_err, 0, sizeof(int), E->stream) != cudaSuccess) rc = SLCS_ERR_CUDA;
    if (rc == SLCS_OK && cudaStreamSynchronize(E->stream) != cudaSuccess) rc = fail(SLCS_ERR_CUDA, "plan setup failed");
    if (rc != SLCS_OK) {
        slcs_sa_plan_destroy(h);
        return rc;
    }
    *out = h;
    return SLCS_OK;
}

int slcs_sa_plan_run(slcs_sa_plan *h, const int32_t *d_p, const int32_t *d_q, int32_t *d_r, int use_graph,
                     void *stream) {
    if (!h) return fail(SLCS_ERR_ARG, "NULL plan");
    if (h->n > 0 && (!d_p || !d_q || !d_r)) return fail(SLCS_ERR_ARG, "NULL buffer");
    SLCS_CUDA_TRY(cudaSetDevice(h->device));
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    if (!use_graph) return sa_plan_run(h->plan, d_p, d_q, d_r, h->d_err, s);
    if (!h->gexec || h->gp != d_p || h->gq != d_q || h->gr != d_r) {
        if (h->gexec) cudaGraphExecDestroy(h->gexec);
        if (h->graph) cudaGraphDestroy(h->graph);
        h->gexec = nullptr;
        h->graph = nullptr;
        cudaStream_t cap;
        SLCS_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        SLCS_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        const int rc = sa_plan_run(h->plan, d_p, d_q, d_r, h->d_err, cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc != SLCS_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return rc != SLCS_OK ? rc : fail(SLCS_ERR_CUDA, std::string("capture failed: ") + cudaGetErrorString(e));
        }
        h->graph = g;
        SLCS_CUDA_TRY(cudaGraphInstantiate(&h->gexec, g, 0));
        h->gp = d_p;
        h->gq = d_q;
        h->gr = d_r;
    }
    SLCS_CUDA_TRY(cudaGraphLaunch(h->gexec, s));
    return SLCS_OK;
}

int slcs_sa_plan_check(slcs_sa_plan *h, void *stream) {
    if (!h) return fail(SLCS_ERR_ARG, "NULL plan");
    Engine *E;
    SLCS_TRY(engine(&E));
    return check_dev_err(h->d_err, stream ? (cudaStream_t) stream : E->stream);
}

int slcs_sa_plan_launches(slcs_sa_plan *h, int32_t *launches) {
    if (!h || !launches) return fail(SLCS_ERR_ARG, "NULL argument");
    *launches = sa_plan_launches(h->plan);
    return SLCS_OK;
}

int slcs_sa_plan_destroy(slcs_sa_plan *h) {
    if (!h) return SLCS_OK;
    cudaSetDevice(h->device);
    Engine *E = nullptr;
    if (engine(&E) == SLCS_OK) cudaStreamSynchronize(E->stream);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->plan) sa_plan_destroy(h->plan);
    if (h->d_err) dfree(h->d_err, E ? E->stream : nullptr);
    if (E) cudaStreamSynchronize(E->stream);
    delete h;
    return SLCS_OK;
}

int slcs_steady_ant(const int32_t *p, const int32_t *q, int n, int32_t *r, const slcs_opts *opts) {
    if (n < 0) return fail(SLCS_ERR_ARG, "negative size");
    if (n > 0 && (!p || !q || !r)) return fail(SLCS_ERR_ARG, "NULL buffer");
    if (n >= (1 << 30)) return fail(SLCS_ERR_TOO_LARGE, "n must be below 2^30");
    Engine *E;
    SLCS_TRY(engine(&E));
    if (n == 0) return SLCS_OK;
    cudaStream_t s = E->stream;
    DevBuf<int32_t> dp, dq, dr;
    SLCS_TRY(dp.alloc(n, s));
    SLCS_TRY(dq.alloc(n, s));
    SLCS_TRY(dr.alloc(n, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dp.p, p, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dq.p, q, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
    SLCS_TRY(slcs_steady_ant_dev(dp.p, dq.p, n, dr.p, opts, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(r, dr.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    return SLCS_OK;
}

}  // extern "C"
