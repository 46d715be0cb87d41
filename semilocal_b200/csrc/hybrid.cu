// hybrid.cu -- the hybrid semi-local scheme on sm_100a: tiles combed independently, braids glued by steady ant.
//
// Follows the reference's iterative hybrid (R:include/SemiLocal/SemiLocalLCS.h:602-792): a grid of M x N tiles
// is combed (each tile a separate braid with its own strand numbering), then the braids are glued pairwise in
// ceil(log2 N) + ceil(log2 M) reduction steps that alternate between joining horizontal neighbours (row
// reduction: the k = rows shared strands are the left braid's right exits / the right braid's left entries)
// and vertical neighbours (column reduction, k = columns), chosen by the same rule (:719-723).  A glue is the
// reference's staggeredStickyMultiplication (R:common/include/Permutations/MongeMultuplicationStrategy.h:
// 679-758): a steady-ant product of the two k x k slices plus the strands that bypass the shared boundary.
//
// On the GPU every step is batched: all tiles go through one persistent combing launch, and each reduction
// step runs three kernels over all its glues (gather the slices, batched steady ant, scatter the product)
// plus a copy of the braids that have no partner.  The slices need no compaction: the steady ant only
// compares ids, so it takes the strands' own row / column ids, and the sorted lists at its root are exactly
// the reference's row and column mappers.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

constexpr int kHT = 2048;   // elements per CTA tile of the gather / scatter kernels

struct GlueDesc {
    int64_t p_off, q_off, out_off, sa_off;
    int psz, qsz, k, row_glue;
};

struct CarryDesc {
    int64_t src, dst;
    int size, pad;
};

struct GTile {
    int g;   // glue (or carry) index
    int t;   // tile inside it
};

// Steady-ant leaves of every glue: for common index j, the id of the left braid's strand that ends at its
// j-th shared exit and the id of the right/lower braid's exit of the strand entering at its j-th shared entry.
__global__ void glue_gather_kernel(const GlueDesc *__restrict__ glues, const GTile *__restrict__ tiles,
                                   const int32_t *__restrict__ r2c, const int32_t *__restrict__ c2r,
                                   int32_t *__restrict__ leafP, int32_t *__restrict__ leafQ) {
    const GTile tl = tiles[blockIdx.x];
    const GlueDesc G = glues[tl.g];
    const int j0 = tl.t * kHT, j1 = min(j0 + kHT, G.k);
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        if (G.row_glue) {   // p above q: p's bottom exits [0, k) feed q's top entries [qsz - k, qsz)
            leafP[G.sa_off + j] = c2r[G.p_off + j];
            leafQ[G.sa_off + j] = r2c[G.q_off + (G.qsz - G.k) + j];
        } else {            // p left of q: p's right exits [psz - k, psz) feed q's left entries [0, k)
            leafP[G.sa_off + j] = c2r[G.p_off + (G.psz - G.k) + j];
            leafQ[G.sa_off + j] = r2c[G.q_off + j];
        }
    }
}

// The glued braid: the steady-ant product for the strands crossing the shared boundary, the others copied
// with their new numbering (R:common/include/Permutations/MongeMultuplicationStrategy.h:726-755).
__global__ void glue_scatter_kernel(const GlueDesc *__restrict__ glues, const GTile *__restrict__ tiles,
                                    const int32_t *__restrict__ r2c, const int32_t *__restrict__ c2r,
                                    const int32_t *__restrict__ PL, const int32_t *__restrict__ QL,
                                    const int32_t *__restrict__ RES, int32_t *__restrict__ out_r2c,
                                    int32_t *__restrict__ out_c2r, int *err) {
    const GTile tl = tiles[blockIdx.x];
    const GlueDesc G = glues[tl.g];
    const int osz = G.psz + G.qsz - G.k;
    const int t0 = tl.t * kHT, t1 = min(t0 + kHT, osz);
    for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
        int row, col;
        if (t < G.k) {
            const int rc = RES[G.sa_off + t];
            if (rc < 0 || rc >= G.k) {
                raise_error(err, kDevErrBadState);
                continue;
            }
            const int prow = PL[G.sa_off + t], qcol = QL[G.sa_off + rc];
            if (G.row_glue) {
                row = G.qsz - G.k + prow;
                col = qcol;
            } else {
                row = prow;
                col = qcol + G.psz - G.k;
            }
        } else if (t < G.psz) {   // strands of p that do not cross into q
            const int j = G.row_glue ? t : t - G.k;
            const int r0 = c2r[G.p_off + j];
            if (G.row_glue) {
                row = r0 + G.qsz - G.k;
                col = j + G.qsz - G.k;
            } else {
                row = r0;
                col = j;
            }
        } else {                  // strands of q that do not come from p
            const int i = G.row_glue ? t - G.psz : t - G.psz + G.k;
            const int c0 = r2c[G.q_off + i];
            if (G.row_glue) {
                row = i;
                col = c0;
            } else {
                row = i - G.k + G.psz;
                col = G.psz - G.k + c0;
            }
        }
        if (row < 0 || row >= osz || col < 0 || col >= osz) {
            raise_error(err, kDevErrBadState);
            continue;
        }
        out_r2c[G.out_off + row] = col;
        out_c2r[G.out_off + col] = row;
    }
}

__global__ void carry_kernel(const CarryDesc *__restrict__ carries, const GTile *__restrict__ tiles,
                             const int32_t *__restrict__ r2c, const int32_t *__restrict__ c2r,
                             int32_t *__restrict__ out_r2c, int32_t *__restrict__ out_c2r) {
    const GTile tl = tiles[blockIdx.x];
    const CarryDesc C = carries[tl.g];
    const int t0 = tl.t * kHT, t1 = min(t0 + kHT, C.size);
    for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
        out_r2c[C.dst + t] = r2c[C.src + t];
        out_c2r[C.dst + t] = c2r[C.src + t];
    }
}

// c2r -> r2c of every tile braid (tile p occupies [off[p], off[p+1]))
__global__ void tiles_invert_kernel(const int32_t *__restrict__ c2r, const int64_t *__restrict__ off,
                                    int32_t *__restrict__ r2c, int *err) {
    const int p = blockIdx.x;
    const int64_t o = off[p];
    const int size = (int) (off[p + 1] - o);
    for (int i = threadIdx.x; i < size; i += blockDim.x) {
        const int r = c2r[o + i];
        if (r < 0 || r >= size) {
            raise_error(err, kDevErrBadState);
            continue;
        }
        r2c[o + r] = i;
    }
}

__global__ void global_score_kernel(const int32_t *__restrict__ c2r, int m, int n, int32_t *score) {
    int cnt = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) cnt += c2r[c] < m;
    cnt = __reduce_add_sync(kFull, cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(score, cnt);
}

struct Block {
    int64_t off;
    int m, n;
};

struct GlueLevel {
    int nglues = 0, ncarries = 0, ngtiles = 0, nstiles = 0, nctiles = 0;
    GlueDesc *d_glues = nullptr;
    CarryDesc *d_carries = nullptr;
    GTile *d_gtiles = nullptr, *d_stiles = nullptr, *d_ctiles = nullptr;
    SaPlan *sa = nullptr;
    int64_t out_total = 0, sa_total = 0;
};

}  // namespace

struct HybridPlan {
    int m = 0, n = 0, M = 0, N = 0;
    int64_t tile_total = 0;
    // tiles
    std::vector<CombItem> items;
    std::vector<int> prog_first;   // tile t's progress slots start here
    CombPair *d_pairs = nullptr;
    CombItem *d_items = nullptr;
    int64_t *d_tile_off = nullptr;
    int32_t *d_prog = nullptr;
    int *d_next = nullptr;
    int nprog = 0;
    int resident = 0;
    // ping-pong braid buffers
    int32_t *r2c[2] = {nullptr, nullptr}, *c2r[2] = {nullptr, nullptr};
    int64_t buf_elems = 0;
    // steady-ant leaves / roots
    int32_t *leafP = nullptr, *leafQ = nullptr, *PL = nullptr, *QL = nullptr, *RES = nullptr;
    SaScratch scratch;
    std::vector<GlueLevel> levels;
    int final_buf = 0;
    cudaStream_t s = nullptr;
    const void *bound_a = nullptr, *bound_b = nullptr;
    std::vector<CombPair> pairs_host;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;   // around the tile combing launch (optional)
    bool capturing = false;
};

void hybrid_plan_destroy(HybridPlan *H) {
    if (!H) return;
    if (H->ev0) cudaEventDestroy(H->ev0);
    if (H->ev1) cudaEventDestroy(H->ev1);
    cudaStream_t s = H->s;
    for (GlueLevel &L : H->levels) {
        void *ps[] = {L.d_glues, L.d_carries, L.d_gtiles, L.d_stiles, L.d_ctiles};
        for (void *p : ps) dfree(p, s);
        if (L.sa) sa_plan_destroy(L.sa);
    }
    void *ps[] = {H->d_pairs, H->d_items, H->d_tile_off, H->d_prog, H->d_next, H->r2c[0], H->r2c[1], H->c2r[0],
                  H->c2r[1], H->leafP, H->leafQ, H->PL, H->QL, H->RES, H->scratch.tabp, H->scratch.vecp,
                  H->scratch.cstp};
    for (void *p : ps) dfree(p, s);
    for (int i = 0; i < 11; ++i) dfree(H->scratch.b[i], s);
    delete H;
}

void hybrid_plan_set_stream(HybridPlan *H, cudaStream_t s) {
    if (!H) return;
    H->s = s;
    for (GlueLevel &L : H->levels) sa_plan_set_stream(L.sa, s);
}

namespace {
template <typename T>
int up(T **dst, const std::vector<T> &v, cudaStream_t s) {
    SLCS_TRY(dalloc(reinterpret_cast<void **>(dst), sizeof(T) * std::max<size_t>(v.size(), 1), s));
    if (!v.empty()) SLCS_CUDA_TRY(cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
    return SLCS_OK;
}
void add_tiles(std::vector<GTile> &v, int g, int64_t len) {
    for (int t = 0; (int64_t) t * kHT < len; ++t) v.push_back(GTile{g, t});
}
}  // namespace

// Plans the hybrid for an m x n grid with tiles of at most tile_rows x tile_cols.
int hybrid_plan_create(int m, int n, int tile_rows, int tile_cols, Engine *E, cudaStream_t s, HybridPlan **out) {
    *out = nullptr;
    auto H = new HybridPlan();
    H->m = m;
    H->n = n;
    H->s = s;
    auto bail = [&](int rc) {
        hybrid_plan_destroy(H);
        return rc;
    };
    // tile grid: the fewest tiles of at most tile_rows x tile_cols, sizes balanced (the reference's
    // rowsPerBlock / colsPerBlock, R:include/SemiLocal/SemiLocalLCS.h:619-627, 663-666)
    const int M = (m + tile_rows - 1) / tile_rows, N = (n + tile_cols - 1) / tile_cols;
    const int rpb = (m + M - 1) / M, cpb = (n + N - 1) / N;
    H->M = (m + rpb - 1) / rpb;
    H->N = (n + cpb - 1) / cpb;
    std::vector<Block> cur;
    std::vector<int64_t> tile_off;
    int64_t acc = 0;
    for (int i = 0; i < H->M; ++i)
        for (int j = 0; j < H->N; ++j) {
            const int r0 = i * rpb, c0 = j * cpb;
            const int mt = std::min(rpb, m - r0), nt = std::min(cpb, n - c0);
            cur.push_back(Block{acc, mt, nt});
            tile_off.push_back(acc);
            acc += mt + nt;
        }
    tile_off.push_back(acc);
    H->tile_total = acc;
    H->pairs_host.resize(cur.size());
    int nprog = 0;
    for (size_t t = 0; t < cur.size(); ++t) {
        H->pairs_host[t] = CombPair{nullptr, nullptr, nullptr, nullptr, nullptr, cur[t].m, cur[t].n};
        nprog += plan_bands((int) t, cur[t].m, pick_rows_batch(cur[t].m), H->items);
    }
    H->nprog = nprog;
    // band-major order: a tile's band k is taken once its band k-1 is under way (progress slots do not depend
    // on the order: tile t's slots start at the number of bands of the tiles before it)
    H->prog_first.assign(cur.size() + 1, 0);
    for (const CombItem &it : H->items) H->prog_first[it.pair + 1]++;
    for (size_t t = 0; t < cur.size(); ++t) H->prog_first[t + 1] += H->prog_first[t];
    std::stable_sort(H->items.begin(), H->items.end(), [](const CombItem &x, const CombItem &y) { return x.band < y.band; });
    H->resident = comb_resident_warps(E);
    // reduction schedule (R:include/SemiLocal/SemiLocalLCS.h:708-789)
    int smallM = H->M, smallN = H->N;
    int64_t blockRows = rpb, blockCols = cpb;
    const int steps = (int) std::ceil(std::log2((double) smallN)) + (int) std::ceil(std::log2((double) smallM));
    int64_t buf_max = acc, sa_max = 1;
    std::vector<std::vector<int64_t>> sa_offs;
    std::vector<std::vector<int>> sa_ns;
    int64_t need_elems = 1, need_tab = 0, need_vec = 0, need_cst = 0;
    SaScratch deferred;
    deferred.elems = -1;
    for (int st = 0; st < steps; ++st) {
        bool in_row = smallN > smallM;
        if (smallN > 1 && smallM > 1) in_row = blockRows >= 2 * blockCols;
        if (in_row) blockCols *= 2;
        else blockRows *= 2;
        const int newCols = in_row ? (smallN + 1) / 2 : smallN;
        const int newRows = in_row ? smallM : (smallM + 1) / 2;
        std::vector<Block> nxt(newRows * newCols);
        std::vector<GlueDesc> glues;
        std::vector<CarryDesc> carries;
        std::vector<int64_t> so;
        std::vector<int> sn;
        int64_t out_acc = 0, sa_acc = 0;
        for (int i = 0; i < newRows * newCols; ++i) {
            const int cr = i / newCols, cc = i % newCols;
            int pi, qi;
            if (in_row) {
                pi = cr * smallN + 2 * cc;
                qi = 2 * cc + 1 < smallN ? pi + 1 : -1;
            } else {
                pi = 2 * cr * smallN + cc;
                qi = 2 * cr + 1 < smallM ? (2 * cr + 1) * smallN + cc : -1;
            }
            const Block &P = cur[pi];
            if (qi < 0) {
                nxt[i] = Block{out_acc, P.m, P.n};
                carries.push_back(CarryDesc{P.off, out_acc, P.m + P.n, 0});
                out_acc += P.m + P.n;
                continue;
            }
            const Block &Q = cur[qi];
            const int k = in_row ? P.m : P.n;
            const int psz = P.m + P.n, qsz = Q.m + Q.n;
            glues.push_back(GlueDesc{P.off, Q.off, out_acc, sa_acc, psz, qsz, k, in_row ? 0 : 1});
            so.push_back(sa_acc);
            sn.push_back(k);
            nxt[i] = in_row ? Block{out_acc, P.m, P.n + Q.n} : Block{out_acc, P.m + Q.m, P.n};
            out_acc += psz + qsz - k;
            sa_acc += k;
        }
        GlueLevel L;
        L.nglues = (int) glues.size();
        L.ncarries = (int) carries.size();
        L.out_total = out_acc;
        L.sa_total = sa_acc;
        std::vector<GTile> gt, stl, ct;
        for (int g = 0; g < L.nglues; ++g) {
            add_tiles(gt, g, glues[g].k);
            add_tiles(stl, g, (int64_t) glues[g].psz + glues[g].qsz - glues[g].k);
        }
        for (int c = 0; c < L.ncarries; ++c) add_tiles(ct, c, carries[c].size);
        L.ngtiles = (int) gt.size();
        L.nstiles = (int) stl.size();
        L.nctiles = (int) ct.size();
        int rc;
        if ((rc = up(&L.d_glues, glues, s)) || (rc = up(&L.d_carries, carries, s)) || (rc = up(&L.d_gtiles, gt, s)) ||
            (rc = up(&L.d_stiles, stl, s)) || (rc = up(&L.d_ctiles, ct, s))) {
            H->levels.push_back(L);
            return bail(rc);
        }
        if (L.nglues) {
            if ((rc = sa_plan_create(so, sn, &L.sa, s, &deferred))) {
                H->levels.push_back(L);
                return bail(rc);
            }
            int64_t e, t, v, c;
            sa_plan_needs(L.sa, &e, &t, &v, &c);
            need_elems = std::max(need_elems, e);
            need_tab = std::max(need_tab, t);
            need_vec = std::max(need_vec, v);
            need_cst = std::max(need_cst, c);
        }
        H->levels.push_back(L);
        buf_max = std::max(buf_max, out_acc);
        sa_max = std::max(sa_max, sa_acc);
        cur.swap(nxt);
        smallN = newCols;
        smallM = newRows;
    }
    H->final_buf = (int) (H->levels.size() % 2);   // level 0 writes buffer 0; each step flips
    H->buf_elems = buf_max;
    int rc;
    if ((rc = up(&H->d_items, H->items, s)) || (rc = up(&H->d_tile_off, tile_off, s))) return bail(rc);
    if ((rc = dalloc(reinterpret_cast<void **>(&H->d_pairs), sizeof(CombPair) * std::max<size_t>(H->pairs_host.size(), 1), s)) ||
        (rc = dalloc(reinterpret_cast<void **>(&H->d_prog), sizeof(int32_t) * std::max(nprog, 1), s)) ||
        (rc = dalloc(reinterpret_cast<void **>(&H->d_next), sizeof(int), s)))
        return bail(rc);
    for (int b = 0; b < 2; ++b)
        if ((rc = dalloc(reinterpret_cast<void **>(&H->r2c[b]), sizeof(int32_t) * buf_max, s)) ||
            (rc = dalloc(reinterpret_cast<void **>(&H->c2r[b]), sizeof(int32_t) * buf_max, s)))
            return bail(rc);
    int32_t **sabufs[] = {&H->leafP, &H->leafQ, &H->PL, &H->QL, &H->RES};
    for (auto b : sabufs)
        if ((rc = dalloc(reinterpret_cast<void **>(b), sizeof(int32_t) * sa_max, s))) return bail(rc);
    SaScratch &S = H->scratch;
    S.elems = need_elems;
    S.tab = need_tab;
    S.vec = need_vec;
    S.cst = need_cst;
    for (int i = 0; i < 11; ++i)
        if ((rc = dalloc(reinterpret_cast<void **>(&S.b[i]), sizeof(int32_t) * need_elems, s))) return bail(rc);
    if ((rc = dalloc(reinterpret_cast<void **>(&S.tabp), sizeof(int32_t) * std::max<int64_t>(need_tab, 1), s)) ||
        (rc = dalloc(reinterpret_cast<void **>(&S.vecp), sizeof(int32_t) * std::max<int64_t>(need_vec, 1), s)) ||
        (rc = dalloc(reinterpret_cast<void **>(&S.cstp), sizeof(int32_t) * std::max<int64_t>(need_cst, 1), s)))
        return bail(rc);
    for (GlueLevel &L : H->levels)
        if (L.sa && (rc = sa_plan_bind(L.sa, &S))) return bail(rc);
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    *out = H;
    return SLCS_OK;
}

// Runs the plan on device strings d_a (m) / d_b (n): kernels only.  The final braid is left in
// (hybrid_result_r2c, hybrid_result_c2r).
template <typename T>
int hybrid_plan_run(HybridPlan *H, const T *d_a, const T *d_b, int *d_err, cudaStream_t s) {
    NvtxRange nv("slcs: hybrid (tiles + glue tree)");
    if (H->bound_a != d_a || H->bound_b != d_b) {
        // tile descriptors point into the strings: rebuilt when the strings move
        std::vector<CombPair> hp = H->pairs_host;
        int64_t acc = 0;
        for (size_t t = 0; t < hp.size(); ++t) {
            const int i = (int) t / H->N, j = (int) t % H->N;
            const int rpb = (H->m + H->M - 1) / H->M, cpb = (H->n + H->N - 1) / H->N;
            hp[t].a = d_a + (int64_t) i * rpb;
            hp[t].b = d_b + (int64_t) j * cpb;
            hp[t].c2r = H->c2r[0] + acc;
            acc += hp[t].m + hp[t].n;
        }
        // one progress slot per band; tile t's slots start at prog_first[t]
        for (size_t t = 0; t < hp.size(); ++t) hp[t].progress = H->d_prog + H->prog_first[t];
        SLCS_CUDA_TRY(cudaMemcpyAsync(H->d_pairs, hp.data(), sizeof(CombPair) * hp.size(), cudaMemcpyHostToDevice, s));
        SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        H->bound_a = d_a;
        H->bound_b = d_b;
    }
    SLCS_CUDA_TRY(cudaMemsetAsync(H->d_prog, 0, sizeof(int32_t) * std::max(H->nprog, 1), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(H->d_next, 0, sizeof(int), s));
    const unsigned fl = H->capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    if (H->ev0) SLCS_CUDA_TRY(cudaEventRecordWithFlags(H->ev0, s, fl));
    SLCS_TRY(launch_comb<T>(H->d_pairs, H->d_items, (int) H->items.size(), H->d_next, d_err, H->resident, s));
    if (H->ev1) SLCS_CUDA_TRY(cudaEventRecordWithFlags(H->ev1, s, fl));
    tiles_invert_kernel<<<(int) H->pairs_host.size(), 256, 0, s>>>(H->c2r[0], H->d_tile_off, H->r2c[0], d_err);
    SLCS_CUDA_TRY(cudaGetLastError());
    int cur = 0;
    for (GlueLevel &L : H->levels) {
        const int nx = cur ^ 1;
        if (L.nglues) {
            glue_gather_kernel<<<L.ngtiles, 256, 0, s>>>(L.d_glues, L.d_gtiles, H->r2c[cur], H->c2r[cur], H->leafP,
                                                         H->leafQ);
            SLCS_CUDA_TRY(cudaGetLastError());
            SLCS_TRY(sa_plan_run_ex(L.sa, nullptr, H->leafP, H->leafQ, H->RES, H->PL, H->QL, d_err, s));
            glue_scatter_kernel<<<L.nstiles, 256, 0, s>>>(L.d_glues, L.d_stiles, H->r2c[cur], H->c2r[cur], H->PL,
                                                          H->QL, H->RES, H->r2c[nx], H->c2r[nx], d_err);
            SLCS_CUDA_TRY(cudaGetLastError());
        }
        if (L.ncarries) {
            carry_kernel<<<L.nctiles, 256, 0, s>>>(L.d_carries, L.d_ctiles, H->r2c[cur], H->c2r[cur], H->r2c[nx],
                                                   H->c2r[nx]);
            SLCS_CUDA_TRY(cudaGetLastError());
        }
        cur = nx;
    }
    H->final_buf = cur;
    return SLCS_OK;
}
template int hybrid_plan_run<uint8_t>(HybridPlan *, const uint8_t *, const uint8_t *, int *, cudaStream_t);
template int hybrid_plan_run<int32_t>(HybridPlan *, const int32_t *, const int32_t *, int *, cudaStream_t);

int32_t *hybrid_result_r2c(HybridPlan *H) { return H->r2c[H->final_buf]; }
int32_t *hybrid_result_c2r(HybridPlan *H) { return H->c2r[H->final_buf]; }

int hybrid_score(HybridPlan *H, int32_t *d_score, cudaStream_t s) {
    SLCS_CUDA_TRY(cudaMemsetAsync(d_score, 0, sizeof(int32_t), s));
    global_score_kernel<<<std::max(1, std::min(1024, (H->n + 255) / 256)), 256, 0, s>>>(hybrid_result_c2r(H), H->m,
                                                                                        H->n, d_score);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}

int hybrid_enable_timing(HybridPlan *H) {
    if (!H->ev0) SLCS_CUDA_TRY(cudaEventCreate(&H->ev0));
    if (!H->ev1) SLCS_CUDA_TRY(cudaEventCreate(&H->ev1));
    return SLCS_OK;
}
void hybrid_set_capturing(HybridPlan *H, bool c) { H->capturing = c; }
int hybrid_comb_ms(HybridPlan *H, float *ms) {
    if (!H->ev0) return fail(SLCS_ERR_ARG, "timing not enabled");
    SLCS_CUDA_TRY(cudaEventSynchronize(H->ev1));
    SLCS_CUDA_TRY(cudaEventElapsedTime(ms, H->ev0, H->ev1));
    return SLCS_OK;
}

int hybrid_launches(const HybridPlan *H) {
    int c = 2;
    for (const GlueLevel &L : H->levels) c += (L.nglues ? 2 + sa_plan_launches(L.sa) : 0) + (L.ncarries ? 1 : 0);
    return c;
}

}  // namespace slcs

using namespace slcs;

extern "C" int slcs_staggered_glue(const int32_t *p, int pm, int pn, const int32_t *q, int qm, int qn, int row_glue,
                                   int32_t *out) {
    if (pm < 0 || pn < 0 || qm < 0 || qn < 0 || !p || !q || !out) return fail(SLCS_ERR_ARG, "bad glue arguments");
    if ((long long) pm + pn + qm + qn >= (1ll << 30))
        return fail(SLCS_ERR_TOO_LARGE, "the braids' strands must number below 2^30");
    const int k = row_glue ? pn : pm;
    if (row_glue ? (qn != pn) : (qm != pm)) return fail(SLCS_ERR_ARG, "the braids do not share k strands");
    const int psz = pm + pn, qsz = qm + qn;
    if (k == psz && k == qsz) return fail(SLCS_ERR_ARG, "the braids have no strands besides the shared ones");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    const int osz = psz + qsz - k;
    DevBuf<int32_t> dp, dq, dpc, dqc, lp, lq, pl, ql, res, o_r, o_c;
    DevBuf<int> err;
    DevBuf<int64_t> offs;
    DevBuf<GlueDesc> dg;
    DevBuf<GTile> gt, stl;
    SLCS_TRY(dp.alloc(psz, s));
    SLCS_TRY(dq.alloc(qsz, s));
    SLCS_TRY(dpc.alloc(psz, s));
    SLCS_TRY(dqc.alloc(qsz, s));
    SLCS_TRY(lp.alloc(k, s));
    SLCS_TRY(lq.alloc(k, s));
    SLCS_TRY(pl.alloc(k, s));
    SLCS_TRY(ql.alloc(k, s));
    SLCS_TRY(res.alloc(k, s));
    SLCS_TRY(o_r.alloc(osz, s));
    SLCS_TRY(o_c.alloc(osz, s));
    SLCS_TRY(err.alloc(1, s));
    SLCS_TRY(offs.alloc(3, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dp.p, p, sizeof(int32_t) * psz, cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dq.p, q, sizeof(int32_t) * qsz, cudaMemcpyHostToDevice, s));
    // column -> row maps of both braids (laid out as two consecutive "tiles": p then q)
    std::vector<int64_t> ho{0, psz, psz + qsz};
    DevBuf<int32_t> both_r2c, both_c2r;
    SLCS_TRY(both_r2c.alloc(psz + qsz, s));
    SLCS_TRY(both_c2r.alloc(psz + qsz, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(both_r2c.p, p, sizeof(int32_t) * psz, cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(both_r2c.p + psz, q, sizeof(int32_t) * qsz, cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(offs.p, ho.data(), sizeof(int64_t) * 3, cudaMemcpyHostToDevice, s));
    // r2c -> c2r: the inversion kernel maps values of one array to indices of the other, either direction
    tiles_invert_kernel<<<2, 256, 0, s>>>(both_r2c.p, offs.p, both_c2r.p, err.p);
    SLCS_CUDA_TRY(cudaGetLastError());
    std::vector<GlueDesc> g{GlueDesc{0, psz, 0, 0, psz, qsz, k, row_glue ? 1 : 0}};
    std::vector<GTile> gtv, stv;
    add_tiles(gtv, 0, k);
    add_tiles(stv, 0, osz);
    SLCS_TRY(up(&dg.p, g, s));
    SLCS_TRY(up(&gt.p, gtv, s));
    SLCS_TRY(up(&stl.p, stv, s));
    dg.s = gt.s = stl.s = s;
    if (k > 0) {
        glue_gather_kernel<<<(int) gtv.size(), 256, 0, s>>>(dg.p, gt.p, both_r2c.p, both_c2r.p, lp.p, lq.p);
        SLCS_CUDA_TRY(cudaGetLastError());
        SaPlan *P = nullptr;
        SLCS_TRY(sa_plan_create(std::vector<int64_t>{0}, std::vector<int>{k}, &P, s, nullptr));
        int rc = sa_plan_run_ex(P, nullptr, lp.p, lq.p, res.p, pl.p, ql.p, err.p, s);
        sa_plan_destroy(P);
        SLCS_TRY(rc);
    }
    glue_scatter_kernel<<<(int) stv.size(), 256, 0, s>>>(dg.p, stl.p, both_r2c.p, both_c2r.p, pl.p, ql.p, res.p, o_r.p,
                                                          o_c.p, err.p);
    SLCS_CUDA_TRY(cudaGetLastError());
    SLCS_CUDA_TRY(cudaMemcpyAsync(out, o_r.p, sizeof(int32_t) * osz, cudaMemcpyDeviceToHost, s));
    return check_dev_err(err.p, s);
}
