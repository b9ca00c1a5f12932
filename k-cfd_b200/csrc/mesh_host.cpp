// Host-side mesh builder of libkcfd: face discovery, geometry, boundary tagging,
// canonical CSR pattern, face -> CSR slot map, face and cell colourings.
//
// Semantics follow the K-CFD reference builder (mesh/mesh_reader.py):
//  * a face id is the rank of the face's first discovery while cells are visited in
//    order and, per cell, edges (2D, :189-214) or the given face lists (3D, :269-290);
//    owner = first cell, neighbour = the last later cell;
//  * 2D geometry :66-78 and :102-113, 3D geometry :81-99 and :116-138 (node-mean
//    centres, Newell normals, divergence-theorem volumes), with the reference's
//    operation order so results agree to the last bit;
//  * boundary tagging :216-231 / :298-313 (last patch assignment of a key wins).
// Face discovery keys every face item by its sorted node tuple (<= 4 nodes, node ids
// < 2^32), buckets the items by their smallest node and matches them inside each
// bucket; face ids are then numbered in item order. The passes that are independent
// per cell, item, face or row run on host threads over fixed chunks, so the result
// is the same bit for bit whatever the thread count; the greedy colourings and the
// neighbour assignment (the last later cell wins) stay sequential.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

#include "kcfd_common.h"

namespace kcfd {

static thread_local std::string g_err;
void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}
const std::string& last_error() { return g_err; }

namespace {

struct Key {
    uint64_t hi, lo;
    bool operator==(const Key& o) const { return hi == o.hi && lo == o.lo; }
};

inline uint64_t mix(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

// Sorted node tuple (k <= 4 nodes, ids < 2^32) packed in 128 bits; unused slots are
// 0xffffffff so faces of different sizes never collide.
inline Key make_key(const int64_t* nodes, int k) {
    uint32_t v[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
    for (int i = 0; i < k; ++i) v[i] = (uint32_t)nodes[i];
    std::sort(v, v + k);
    Key key;
    key.hi = ((uint64_t)v[0] << 32) | v[1];
    key.lo = ((uint64_t)v[2] << 32) | v[3];
    return key;
}

class KeyTable {
   public:
    explicit KeyTable(size_t n_expected) {
        size_t cap = 16;
        while (cap < 2 * n_expected + 16) cap <<= 1;
        mask_ = cap - 1;
        keys_.resize(cap);
        vals_.assign(cap, -1);
    }
    // Returns the slot; *found tells whether the key was present.
    size_t find_or_insert(const Key& k, bool* found) {
        size_t h = (size_t)(mix(k.hi ^ mix(k.lo))) & mask_;
        while (true) {
            if (vals_[h] < 0) {
                keys_[h] = k;
                *found = false;
                return h;
            }
            if (keys_[h] == k) {
                *found = true;
                return h;
            }
            h = (h + 1) & mask_;
        }
    }
    int64_t& val(size_t slot) { return vals_[slot]; }
    int64_t lookup(const Key& k) const {
        size_t h = (size_t)(mix(k.hi ^ mix(k.lo))) & mask_;
        while (true) {
            if (vals_[h] < 0) return -1;
            if (keys_[h] == k) return vals_[h];
            h = (h + 1) & mask_;
        }
    }

   private:
    size_t mask_;
    std::vector<Key> keys_;
    std::vector<int64_t> vals_;
};

// Allocator whose resize() leaves new elements default-initialised (no zero fill):
// the builder writes every element of these arrays on its worker threads.
template <class T>
struct DefaultInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = DefaultInitAlloc<U>;
    };
    DefaultInitAlloc() = default;
    template <class U>
    DefaultInitAlloc(const DefaultInitAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new ((void*)p) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};
template <class T>
using dvec = std::vector<T, DefaultInitAlloc<T>>;

}  // namespace
}  // namespace kcfd

struct kcfd_host_mesh {
    int ndim = 2;
    int64_t n_cells = 0, n_faces = 0, n_internal = 0, nnz = 0;
    int max_face_nodes = 2, max_cell_faces = 0;
    int n_int_colors = 0, n_bnd_colors = 0, n_cell_colors = 0, n_levels = 0;
    kcfd::dvec<int64_t> owner, neighbour, face_nodes, cell_faces;
    kcfd::dvec<double> area, normal, fcenter, ccenter, volume;
    kcfd::dvec<int32_t> face_patch, indptr, indices, slot_on, slot_no, diag_slot;
    kcfd::dvec<int32_t> face_color, cell_color, level_natural;
};

using kcfd::Key;
using kcfd::make_key;
using kcfd::KeyTable;
using kcfd::dvec;

namespace {

// Host threads for the builder's independent passes (per cell, item, face or row):
// KCFD_HOST_THREADS when set (a positive count), else the hardware's, at most 16.
// Read once per process.
int host_threads() {
    static const int t = [] {
        unsigned h = std::thread::hardware_concurrency();
        if (const char* e = std::getenv("KCFD_HOST_THREADS")) {
            const long v = std::strtol(e, nullptr, 10);
            if (v > 0) h = (unsigned)std::min(v, 1024L);
        }
        return (int)std::min(16u, std::max(1u, h));
    }();
    return t;
}

// Chunks of at least 32768 elements, at most one per host thread.
int n_chunks(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(host_threads(), n / 32768)); }

// Runs fn(chunk, begin, end) over `chunks` contiguous pieces of [0, n). The pieces
// depend only on n and chunks, and each element is computed by the same arithmetic
// whatever thread runs it, so results do not depend on the thread count or timing.
// A piece whose thread cannot be started runs on the calling thread.
template <class Fn>
void parallel_chunks(int64_t n, int chunks, Fn&& fn) {
    auto run = [&](int t) { fn(t, n * t / chunks, n * (t + 1) / chunks); };
    std::vector<std::thread> pool;
    int t = 1;
    try {
        for (; t < chunks; ++t) pool.emplace_back(run, t);
    } catch (...) {
    }
    for (int u = t; u < chunks; ++u) run(u);
    run(0);
    for (auto& th : pool) th.join();
}

void build_pattern(kcfd_host_mesh* m) {
    const int64_t n = m->n_cells, F = m->n_faces;
    std::vector<int64_t> cnt(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) cnt[i + 1] += 1;
    for (int64_t f = 0; f < F; ++f)
        if (m->neighbour[f] >= 0) {
            cnt[m->owner[f] + 1] += 1;
            cnt[m->neighbour[f] + 1] += 1;
        }
    for (int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    dvec<int32_t> cols(cnt[n]);
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int64_t i = 0; i < n; ++i) cols[pos[i]++] = (int32_t)i;
    for (int64_t f = 0; f < F; ++f)
        if (m->neighbour[f] >= 0) {
            int64_t o = m->owner[f], nb = m->neighbour[f];
            cols[pos[o]++] = (int32_t)nb;
            cols[pos[nb]++] = (int32_t)o;
        }
    // each row sorted and deduplicated in place, then packed
    dvec<int64_t> ulen(n);
    const int RC = n_chunks(n);
    parallel_chunks(n, RC, [&](int, int64_t r0, int64_t r1) {
        for (int64_t i = r0; i < r1; ++i) {
            auto b = cols.begin() + cnt[i], e = cols.begin() + cnt[i + 1];
            std::sort(b, e);
            ulen[i] = std::unique(b, e) - b;
        }
    });
    m->indptr.resize(n + 1);
    m->indptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) m->indptr[i + 1] = (int32_t)(m->indptr[i] + ulen[i]);
    m->nnz = m->indptr[n];
    m->indices.resize(m->nnz);
    parallel_chunks(n, RC, [&](int, int64_t r0, int64_t r1) {
        for (int64_t i = r0; i < r1; ++i)
            std::copy(cols.begin() + cnt[i], cols.begin() + cnt[i] + ulen[i], m->indices.begin() + m->indptr[i]);
    });
    auto slot = [&](int64_t r, int64_t c) -> int32_t {
        auto b = m->indices.begin() + m->indptr[r], e = m->indices.begin() + m->indptr[r + 1];
        auto it = std::lower_bound(b, e, (int32_t)c);
        return (int32_t)(it - m->indices.begin());
    };
    m->diag_slot.resize(n);
    parallel_chunks(n, RC, [&](int, int64_t r0, int64_t r1) {
        for (int64_t i = r0; i < r1; ++i) m->diag_slot[i] = slot(i, i);
    });
    m->slot_on.resize(F);
    m->slot_no.resize(F);
    parallel_chunks(F, n_chunks(F), [&](int, int64_t f0, int64_t f1) {
        for (int64_t f = f0; f < f1; ++f) {
            const bool in = m->neighbour[f] >= 0;
            m->slot_on[f] = in ? slot(m->owner[f], m->neighbour[f]) : -1;
            m->slot_no[f] = in ? slot(m->neighbour[f], m->owner[f]) : -1;
        }
    });
}

// Greedy edge colouring of internal faces in face order (no two faces of a colour
// share a cell), and per-owner counting colours for boundary faces.
int color_faces(kcfd_host_mesh* m) {
    const int64_t n = m->n_cells, F = m->n_faces;
    std::vector<uint64_t> used(n, 0);
    m->face_color.assign(F, -1);
    int ci = 0;
    for (int64_t f = 0; f < F; ++f) {
        if (m->neighbour[f] < 0) continue;
        uint64_t u = used[m->owner[f]] | used[m->neighbour[f]];
        if (~u == 0) return -1;
        int c = __builtin_ctzll(~u);
        used[m->owner[f]] |= 1ULL << c;
        used[m->neighbour[f]] |= 1ULL << c;
        m->face_color[f] = c;
        ci = std::max(ci, c + 1);
    }
    std::vector<int32_t> nb(n, 0);
    int cb = 0;
    for (int64_t f = 0; f < F; ++f) {
        if (m->neighbour[f] >= 0) continue;
        int c = nb[m->owner[f]]++;
        m->face_color[f] = ci + c;
        cb = std::max(cb, c + 1);
    }
    m->n_int_colors = ci;
    m->n_bnd_colors = cb;
    return 0;
}

void color_cells_and_levels(kcfd_host_mesh* m) {
    const int64_t n = m->n_cells;
    m->cell_color.assign(n, -1);
    m->level_natural.assign(n, 0);
    int nc = 0, nl = 0;
    std::vector<char> seen;
    for (int64_t i = 0; i < n; ++i) {
        seen.assign(nc + 1, 0);
        int lev = 0;
        for (int32_t k = m->indptr[i]; k < m->indptr[i + 1]; ++k) {
            int32_t j = m->indices[k];
            if (j == i) continue;
            if (m->cell_color[j] >= 0) seen[m->cell_color[j]] = 1;
            if (j < i) lev = std::max(lev, m->level_natural[j] + 1);
        }
        int c = 0;
        while (c < nc && seen[c]) ++c;
        m->cell_color[i] = c;
        nc = std::max(nc, c + 1);
        m->level_natural[i] = lev;
        nl = std::max(nl, lev + 1);
    }
    m->n_cell_colors = nc;
    m->n_levels = nl;
}

}  // namespace

extern "C" {

int kcfd_mesh_build(int32_t ndim, int64_t n_nodes, const double* nodes, int64_t n_cells,
                    const int64_t* cell_ptr, const int64_t* cell_nodes, const int64_t* cface_ptr,
                    const int64_t* cface_len, const int64_t* cface_off, const int64_t* cface_nodes,
                    int64_t n_bfaces, const int64_t* bface_len, const int64_t* bface_nodes,
                    const int32_t* bface_patch, kcfd_host_mesh** out) {
    KCFD_REQUIRE(out != nullptr, "kcfd_mesh_build: out is NULL");
    *out = nullptr;
    KCFD_REQUIRE(ndim == 2 || ndim == 3, "kcfd_mesh_build: ndim must be 2 or 3 (got %d)", ndim);
    KCFD_REQUIRE(n_nodes > 0 && n_nodes < 0xffffffffLL, "kcfd_mesh_build: bad n_nodes %lld", (long long)n_nodes);
    KCFD_REQUIRE(n_cells > 0 && n_cells < 0x7fffffffLL, "kcfd_mesh_build: bad n_cells %lld", (long long)n_cells);
    KCFD_REQUIRE(nodes && cell_ptr && cell_nodes, "kcfd_mesh_build: NULL node/cell arrays");
    const bool is3d = (ndim == 3 && cface_ptr != nullptr);
    if (ndim == 3) KCFD_REQUIRE(cface_ptr && cface_len && cface_off && cface_nodes, "kcfd_mesh_build: 3D needs cell face lists");
    KCFD_REQUIRE(cell_ptr[0] == 0 && (!is3d || cface_ptr[0] == 0), "kcfd_mesh_build: offsets must start at 0");
    for (int64_t c = 0; c < n_cells; ++c) {
        KCFD_REQUIRE(cell_ptr[c + 1] > cell_ptr[c], "kcfd_mesh_build: cell %lld has no nodes", (long long)c);
        if (is3d) KCFD_REQUIRE(cface_ptr[c + 1] >= cface_ptr[c], "kcfd_mesh_build: cell face offsets decrease at cell %lld", (long long)c);
    }
    for (int64_t k = 0; k < cell_ptr[n_cells]; ++k)
        KCFD_REQUIRE(cell_nodes[k] >= 0 && cell_nodes[k] < n_nodes, "kcfd_mesh_build: cell node %lld out of range", (long long)cell_nodes[k]);

    auto* m = new kcfd_host_mesh();
    m->ndim = ndim;
    m->n_cells = n_cells;
    const int64_t n = n_cells;
    const int D = ndim;
    const int CC = n_chunks(n);
    // ---- cell centres (node mean, sequential sum) and 2D areas (shoelace) ----
    m->ccenter.resize(n * D);
    m->volume.resize(n);  // 2D: shoelace below; 3D: divergence theorem after the faces
    parallel_chunks(n, CC, [&](int, int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1; ++c) {
            int64_t b = cell_ptr[c], e = cell_ptr[c + 1];
            int k = (int)(e - b);
            for (int d = 0; d < D; ++d) {
                double s = nodes[cell_nodes[b] * D + d];
                for (int i = 1; i < k; ++i) s = s + nodes[cell_nodes[b + i] * D + d];
                m->ccenter[c * D + d] = s / (double)k;
            }
            if (!is3d) {
                double a = 0.0;
                for (int i = 0; i < k; ++i) {
                    const double* pi = nodes + cell_nodes[b + i] * D;
                    const double* pj = nodes + cell_nodes[b + (i + 1) % k] * D;
                    double t1 = pi[0] * pj[1];
                    double t2 = pj[0] * pi[1];
                    a = a + (t1 - t2);
                }
                m->volume[c] = std::fabs(a) / 2.0;
            }
        }
    });
    // ---- face discovery ----
    // Every face item (a 2D cell edge or a given 3D face list) gets the key of its
    // sorted node tuple. Items are bucketed by their smallest node id, which keeps
    // the matching local (neighbouring cells share nodes), and matched inside each
    // bucket; an item whose key has no earlier item is the face's first discovery.
    // Face ids then follow item order, which is the reference's visiting order
    // (cells in order, items of a cell in order).
    const int64_t* iptr = is3d ? cface_ptr : cell_ptr;
    const int64_t n_items = iptr[n];
    auto item_nodes = [&](int64_t it, int64_t c, int64_t* buf) -> int {
        if (is3d) {
            int k = (int)cface_len[it];
            for (int i = 0; i < k; ++i) buf[i] = cface_nodes[cface_off[it] + i];
            return k;
        }
        int64_t b = cell_ptr[c], e = cell_ptr[c + 1];
        int64_t pos = it - b;
        buf[0] = cell_nodes[it];
        buf[1] = cell_nodes[b + (pos + 1) % (e - b)];
        return 2;
    };
    dvec<Key> item_key(n_items);
    dvec<int32_t> item_cell(n_items);
    struct ItemError {
        int64_t item = -1;
        int kind = 0, k = 0;
    };
    std::vector<ItemError> err_c(CC);
    std::vector<int> kmax_c(CC, 2);
    parallel_chunks(n, CC, [&](int t, int64_t c0, int64_t c1) {
        int64_t buf[4];
        for (int64_t c = c0; c < c1; ++c)
            for (int64_t it = iptr[c]; it < iptr[c + 1]; ++it) {
                const int k = is3d ? (int)cface_len[it] : 2;
                if (k < 2 || k > 4) {
                    err_c[t] = {it, 1, k};
                    return;
                }
                item_nodes(it, c, buf);
                for (int i = 0; i < k; ++i)
                    if (buf[i] < 0 || buf[i] >= n_nodes) {
                        err_c[t] = {it, 2, k};
                        return;
                    }
                kmax_c[t] = std::max(kmax_c[t], k);
                item_key[it] = make_key(buf, k);
                item_cell[it] = (int32_t)c;
            }
    });
    int kmax_face = 2;
    for (int t = 0; t < CC; ++t) {
        if (err_c[t].item >= 0) {  // the chunks are in item order: this is the first bad item
            delete m;
            if (err_c[t].kind == 1)
                kcfd::set_error("kcfd_mesh_build: faces need 2..4 nodes (got %d)", err_c[t].k);
            else
                kcfd::set_error("kcfd_mesh_build: face node out of range");
            return KCFD_BAD_INPUT;
        }
        kmax_face = std::max(kmax_face, kmax_c[t]);
    }
    std::vector<int64_t> bucket_ptr(n_nodes + 1, 0);
    for (int64_t it = 0; it < n_items; ++it) bucket_ptr[(item_key[it].hi >> 32) + 1] += 1;
    for (int64_t v = 0; v < n_nodes; ++v) bucket_ptr[v + 1] += bucket_ptr[v];
    dvec<int64_t> bucket(n_items);
    {
        std::vector<int64_t> fill(bucket_ptr.begin(), bucket_ptr.end() - 1);
        for (int64_t it = 0; it < n_items; ++it) bucket[fill[item_key[it].hi >> 32]++] = it;
    }
    // rep[it]: the first item with the same key (itself for a first discovery)
    dvec<int64_t> rep(n_items);
    parallel_chunks(n_nodes, n_chunks(n_nodes), [&](int, int64_t v0, int64_t v1) {
        std::vector<int64_t> order;
        for (int64_t v = v0; v < v1; ++v) {
            const int64_t b = bucket_ptr[v], e = bucket_ptr[v + 1];
            if (e - b <= 32) {
                for (int64_t j = b; j < e; ++j) {
                    const int64_t it = bucket[j];
                    int64_t r = it;
                    for (int64_t q = b; q < j; ++q)
                        if (item_key[bucket[q]] == item_key[it]) {
                            r = rep[bucket[q]];
                            break;
                        }
                    rep[it] = r;
                }
            } else {  // a node shared by many faces: sort the bucket by (key, item)
                order.assign(bucket.begin() + b, bucket.begin() + e);
                std::sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
                    const Key& p = item_key[x];
                    const Key& q = item_key[y];
                    if (p.hi != q.hi) return p.hi < q.hi;
                    if (p.lo != q.lo) return p.lo < q.lo;
                    return x < y;
                });
                for (size_t j = 0; j < order.size(); ++j)
                    rep[order[j]] =
                        (j > 0 && item_key[order[j]] == item_key[order[j - 1]]) ? rep[order[j - 1]] : order[j];
            }
        }
    });
    dvec<Key>().swap(item_key);
    dvec<int64_t>().swap(bucket);
    // face ids: first discoveries numbered in item order
    const int IC = n_chunks(n_items);
    std::vector<int64_t> first_off(IC + 1, 0);
    parallel_chunks(n_items, IC, [&](int t, int64_t i0, int64_t i1) {
        int64_t k = 0;
        for (int64_t it = i0; it < i1; ++it) k += (rep[it] == it);
        first_off[t + 1] = k;
    });
    for (int t = 0; t < IC; ++t) first_off[t + 1] += first_off[t];
    const int64_t F = first_off[IC];
    dvec<int64_t> first_item(F);  // per face: item index of first discovery
    dvec<int64_t> item_face(n_items);
    m->owner.resize(F);
    m->neighbour.resize(F);
    parallel_chunks(n_items, IC, [&](int t, int64_t i0, int64_t i1) {
        int64_t f = first_off[t];
        for (int64_t it = i0; it < i1; ++it)
            if (rep[it] == it) {
                item_face[it] = f;
                first_item[f] = it;
                m->owner[f] = item_cell[it];
                m->neighbour[f] = -1;
                ++f;
            }
    });
    parallel_chunks(n_items, IC, [&](int, int64_t i0, int64_t i1) {
        for (int64_t it = i0; it < i1; ++it)
            if (rep[it] != it) item_face[it] = item_face[rep[it]];
    });
    for (int64_t it = 0; it < n_items; ++it)  // in item order: the last later cell wins
        if (rep[it] != it) m->neighbour[item_face[it]] = item_cell[it];
    dvec<int64_t>().swap(rep);
    m->n_faces = F;
    m->max_face_nodes = kmax_face;
    int kc = 0;
    for (int64_t c = 0; c < n; ++c) kc = std::max<int64_t>(kc, iptr[c + 1] - iptr[c]);
    m->max_cell_faces = kc;
    m->cell_faces.resize(n * kc);
    parallel_chunks(n, CC, [&](int, int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1; ++c)
            for (int64_t j = 0; j < kc; ++j)
                m->cell_faces[c * kc + j] = (iptr[c] + j < iptr[c + 1]) ? item_face[iptr[c] + j] : -1;
    });
    const int FC = n_chunks(F);
    m->face_nodes.resize(F * kmax_face);
    dvec<int> fsize(F);
    parallel_chunks(F, FC, [&](int, int64_t f0, int64_t f1) {
        int64_t buf[4];
        for (int64_t f = f0; f < f1; ++f) {
            int k = item_nodes(first_item[f], m->owner[f], buf);
            fsize[f] = k;
            for (int i = 0; i < kmax_face; ++i) m->face_nodes[f * kmax_face + i] = i < k ? buf[i] : -1;
        }
    });
    int64_t ni = 0;
    for (int64_t f = 0; f < F; ++f) ni += (m->neighbour[f] >= 0);
    m->n_internal = ni;
    // ---- face geometry ----
    m->area.resize(F);
    m->normal.resize(F * D);
    m->fcenter.resize(F * D);
    parallel_chunks(F, FC, [&](int, int64_t f0, int64_t f1) {
        for (int64_t f = f0; f < f1; ++f) {
            const int64_t* fn = &m->face_nodes[f * kmax_face];
            double* nr = &m->normal[f * D];
            double* fc = &m->fcenter[f * D];
            const double* cc = &m->ccenter[m->owner[f] * D];
            if (D == 2) {
                const double* p0 = nodes + fn[0] * 2;
                const double* p1 = nodes + fn[1] * 2;
                fc[0] = 0.5 * (p0[0] + p1[0]);
                fc[1] = 0.5 * (p0[1] + p1[1]);
                double dx = p1[0] - p0[0], dy = p1[1] - p0[1];
                double len = std::sqrt(dx * dx + dy * dy);
                nr[0] = dy;
                nr[1] = -dx;
                if (len > 1e-15) {
                    nr[0] = nr[0] / len;
                    nr[1] = nr[1] / len;
                }
                double t0 = fc[0] - cc[0], t1 = fc[1] - cc[1];
                double dot = nr[0] * t0 + nr[1] * t1;
                if (dot < 0) {
                    nr[0] = -nr[0];
                    nr[1] = -nr[1];
                }
                m->area[f] = len;
            } else {
                int k = fsize[f];
                for (int d = 0; d < 3; ++d) {
                    double s = nodes[fn[0] * 3 + d];
                    for (int i = 1; i < k; ++i) s = s + nodes[fn[i] * 3 + d];
                    fc[d] = s / (double)k;
                }
                double nx = 0.0, ny = 0.0, nz = 0.0;
                for (int i = 0; i < k; ++i) {
                    const double* pi = nodes + fn[i] * 3;
                    const double* pj = nodes + fn[(i + 1) % k] * 3;
                    nx = nx + (pi[1] - pj[1]) * (pi[2] + pj[2]);
                    ny = ny + (pi[2] - pj[2]) * (pi[0] + pj[0]);
                    nz = nz + (pi[0] - pj[0]) * (pi[1] + pj[1]);
                }
                double a = std::sqrt(nx * nx + ny * ny + nz * nz);
                nr[0] = nx;
                nr[1] = ny;
                nr[2] = nz;
                if (a > 1e-15) {
                    nr[0] = nr[0] / a;
                    nr[1] = nr[1] / a;
                    nr[2] = nr[2] / a;
                }
                m->area[f] = a * 0.5;
                double dot = nr[0] * (fc[0] - cc[0]) + nr[1] * (fc[1] - cc[1]) + nr[2] * (fc[2] - cc[2]);
                if (dot < 0) {
                    nr[0] = -nr[0];
                    nr[1] = -nr[1];
                    nr[2] = -nr[2];
                }
            }
        }
    });
    if (is3d) {
        parallel_chunks(n, CC, [&](int, int64_t c0, int64_t c1) {
            for (int64_t c = c0; c < c1; ++c) {
                double vol = 0.0;
                const double* cc = &m->ccenter[c * 3];
                for (int j = 0; j < kc; ++j) {
                    int64_t f = m->cell_faces[c * kc + j];
                    if (f < 0) continue;
                    const double* fc = &m->fcenter[f * 3];
                    const double* nr = &m->normal[f * 3];
                    double sgn = 1.0;
                    double tdot = nr[0] * (fc[0] - cc[0]) + nr[1] * (fc[1] - cc[1]) + nr[2] * (fc[2] - cc[2]);
                    if (tdot < 0) sgn = -1.0;
                    double d = fc[0] * nr[0] + fc[1] * nr[1] + fc[2] * nr[2];
                    vol = vol + sgn * d * m->area[f];
                }
                vol = std::fabs(vol) / 3.0;
                if (vol < 1e-30) vol = 1e-30;
                m->volume[c] = vol;
            }
        });
    }
    // ---- boundary tagging ----
    m->face_patch.assign(F, -1);
    {
        KeyTable bt((size_t)std::max<int64_t>(n_bfaces, 1));
        int64_t off = 0;
        for (int64_t q = 0; q < n_bfaces; ++q) {
            int k = (int)bface_len[q];
            if (k >= 2 && k <= 4) {
                Key key = make_key(bface_nodes + off, k);
                bool found;
                size_t s = bt.find_or_insert(key, &found);
                bt.val(s) = bface_patch[q];  // last assignment wins
            }
            off += k;
        }
        for (int64_t f = 0; f < F; ++f) {
            if (m->neighbour[f] >= 0) continue;
            Key key = make_key(&m->face_nodes[f * kmax_face], fsize[f]);
            int64_t p = bt.lookup(key);
            m->face_patch[f] = (p >= 0) ? (int32_t)p : -2;
        }
    }
    build_pattern(m);
    if (color_faces(m) != 0) {
        delete m;
        kcfd::set_error("kcfd_mesh_build: more than 64 face colours");
        return KCFD_BAD_INPUT;
    }
    color_cells_and_levels(m);
    *out = m;
    return KCFD_OK;
}

int kcfd_mesh_device_layout(int32_t ndim, int64_t n_cells, int64_t n_faces, int64_t n_internal,
                            int32_t n_colors, int32_t max_cell_faces, const int64_t* owner,
                            const int64_t* neighbour, const int32_t* face_color, const double* ccenter,
                            const double* fcenter, const double* normal, const double* area,
                            const int32_t* slot_on, const int32_t* slot_no, const int64_t* cell_faces,
                            kcfd_face_layout_t* o) {
    KCFD_REQUIRE(o && owner && neighbour && face_color && ccenter && fcenter && normal && area && slot_on &&
                     slot_no && cell_faces,
                 "kcfd_mesh_device_layout: NULL argument");
    KCFD_REQUIRE(o->order && o->color_ptr && o->owner && o->neigh && o->area && o->normal && o->fcenter && o->gc &&
                     o->dlen && o->dorth && o->slot_on && o->slot_no && o->cf_ptr && o->cf_face,
                 "kcfd_mesh_device_layout: NULL output array");
    KCFD_REQUIRE(ndim == 2 || ndim == 3, "kcfd_mesh_device_layout: ndim must be 2 or 3 (got %d)", ndim);
    KCFD_REQUIRE(n_cells > 0 && n_cells < 0x7fffffffLL && n_faces > 0 && n_faces < 0x7fffffffLL && n_internal >= 0 &&
                     n_internal <= n_faces && n_colors > 0 && max_cell_faces >= 0,
                 "kcfd_mesh_device_layout: bad sizes");
    const int64_t F = n_faces, Fi = n_internal, n = n_cells;
    const int D = ndim, NC = n_colors;
    // ---- faces ordered by colour, by reference id inside a colour (stable counting sort) ----
    const int FC = n_chunks(F);
    std::vector<char> bad(FC, 0);
    std::vector<int64_t> cnt((size_t)FC * NC, 0);
    parallel_chunks(F, FC, [&](int t, int64_t f0, int64_t f1) {
        int64_t* c = &cnt[(size_t)t * NC];
        for (int64_t f = f0; f < f1; ++f) {
            const int32_t k = face_color[f];
            if (k < 0 || k >= NC || owner[f] < 0 || owner[f] >= n || neighbour[f] < -1 || neighbour[f] >= n) {
                bad[t] = 1;
                return;
            }
            ++c[k];
        }
    });
    for (int t = 0; t < FC; ++t)
        KCFD_REQUIRE(!bad[t], "kcfd_mesh_device_layout: face colour, owner or neighbour out of range");
    std::vector<int64_t> start((size_t)FC * NC);
    int64_t run = 0;
    for (int k = 0; k < NC; ++k) {
        o->color_ptr[k] = (int32_t)run;
        for (int t = 0; t < FC; ++t) {
            start[(size_t)t * NC + k] = run;
            run += cnt[(size_t)t * NC + k];
        }
    }
    o->color_ptr[NC] = (int32_t)run;
    parallel_chunks(F, FC, [&](int t, int64_t f0, int64_t f1) {
        int64_t* s = &start[(size_t)t * NC];
        for (int64_t f = f0; f < f1; ++f) o->order[s[face_color[f]]++] = f;
    });
    // ---- per device face: gathers and geometric factors ----
    auto norm = [D](const double* v) {
        double s = v[0] * v[0];
        for (int k = 1; k < D; ++k) s = s + v[k] * v[k];
        return std::sqrt(s);
    };
    std::fill(bad.begin(), bad.end(), 0);
    parallel_chunks(F, FC, [&](int t, int64_t d0, int64_t d1) {
        for (int64_t d = d0; d < d1; ++d) {
            const int64_t f = o->order[d];
            const int64_t ow = owner[f], nb = neighbour[f];
            if ((d < Fi) != (nb >= 0)) {  // internal colours must come first
                bad[t] = 1;
                return;
            }
            o->owner[d] = (int32_t)ow;
            o->area[d] = area[f];
            const double* cp = ccenter + ow * D;
            const double* fc = fcenter + f * D;
            const double* nr = normal + f * D;
            double eO[3];
            for (int k = 0; k < D; ++k) {
                o->normal[d * D + k] = nr[k];
                o->fcenter[d * D + k] = fc[k];
                eO[k] = fc[k] - cp[k];
            }
            const double dO = norm(eO);
            if (d >= Fi) {
                o->dlen[d] = dO;
                continue;
            }
            o->neigh[d] = (int32_t)nb;
            o->slot_on[d] = slot_on[f];
            o->slot_no[d] = slot_no[f];
            const double* cn = ccenter + nb * D;
            double dv[3], eN[3];
            for (int k = 0; k < D; ++k) {
                dv[k] = cn[k] - cp[k];
                eN[k] = fc[k] - cn[k];
            }
            const double dint = norm(dv);
            double dn = dv[0] * nr[0];
            for (int k = 1; k < D; ++k) dn = dn + dv[k] * nr[k];
            const double a = std::fabs(dn), b = 0.1 * dint;
            o->dorth[d] = (a != a) ? a : (b != b) ? b : (a >= b ? a : b);  // NaN-propagating max
            o->dlen[d] = dint;
            const double dN = norm(eN), sum = dO + dN;
            o->gc[d] = (sum > 1e-30) ? dN / sum : 0.5;
        }
    });
    for (int t = 0; t < FC; ++t)
        KCFD_REQUIRE(!bad[t], "kcfd_mesh_device_layout: internal faces must take the first colours");
    // ---- faces of each cell, ascending reference id, as device indices ----
    std::vector<int32_t> dev_of_ref(F);
    parallel_chunks(F, FC, [&](int, int64_t d0, int64_t d1) {
        for (int64_t d = d0; d < d1; ++d) dev_of_ref[o->order[d]] = (int32_t)d;
    });
    const int kc = max_cell_faces, CC = n_chunks(n);
    std::vector<int32_t> nvalid(n);
    std::vector<char> badc(CC, 0);
    parallel_chunks(n, CC, [&](int t, int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1; ++c) {
            int k = 0;
            for (int j = 0; j < kc; ++j) {
                const int64_t v = cell_faces[c * kc + j];
                if (v >= F) {
                    badc[t] = 1;
                    return;
                }
                k += (v >= 0);
            }
            nvalid[c] = k;
        }
    });
    for (int t = 0; t < CC; ++t) KCFD_REQUIRE(!badc[t], "kcfd_mesh_device_layout: cell face id out of range");
    int64_t total = 0;
    o->cf_ptr[0] = 0;
    for (int64_t c = 0; c < n; ++c) {
        total += nvalid[c];
        KCFD_REQUIRE(total < 0x7fffffffLL, "kcfd_mesh_device_layout: too many cell faces");
        o->cf_ptr[c + 1] = (int32_t)total;
    }
    parallel_chunks(n, CC, [&](int, int64_t c0, int64_t c1) {
        std::vector<int64_t> tmp(kc > 0 ? kc : 1);
        for (int64_t c = c0; c < c1; ++c) {
            int m = 0;
            for (int j = 0; j < kc; ++j)
                if (cell_faces[c * kc + j] >= 0) tmp[m++] = cell_faces[c * kc + j];
            std::sort(tmp.begin(), tmp.begin() + m);
            for (int i = 0; i < m; ++i) o->cf_face[o->cf_ptr[c] + i] = dev_of_ref[tmp[i]];
        }
    });
    return KCFD_OK;
}

int kcfd_mesh_info(const kcfd_host_mesh* m, int64_t* info) {
    KCFD_REQUIRE(m && info, "kcfd_mesh_info: NULL argument");
    info[0] = m->n_faces;
    info[1] = m->n_internal;
    info[2] = m->nnz;
    info[3] = m->max_face_nodes;
    info[4] = m->max_cell_faces;
    info[5] = m->n_int_colors;
    info[6] = m->n_bnd_colors;
    info[7] = m->n_cell_colors;
    info[8] = m->n_levels;
    info[9] = m->ndim;
    return KCFD_OK;
}

int kcfd_mesh_export(const kcfd_host_mesh* m, kcfd_mesh_export_t* o) {
    KCFD_REQUIRE(m && o, "kcfd_mesh_export: NULL argument");
    auto cp = [](auto* dst, const auto& v) {
        if (!dst) return;
        const int64_t bytes = (int64_t)(v.size() * sizeof(v[0]));
        char* d = reinterpret_cast<char*>(dst);
        const char* s = reinterpret_cast<const char*>(v.data());
        parallel_chunks(bytes, n_chunks(bytes / 64), [&](int, int64_t b, int64_t e) { std::memcpy(d + b, s + b, e - b); });
    };
    cp(o->owner, m->owner);
    cp(o->neighbour, m->neighbour);
    cp(o->face_nodes, m->face_nodes);
    cp(o->cell_faces, m->cell_faces);
    cp(o->area, m->area);
    cp(o->normal, m->normal);
    cp(o->fcenter, m->fcenter);
    cp(o->ccenter, m->ccenter);
    cp(o->volume, m->volume);
    cp(o->face_patch, m->face_patch);
    cp(o->indptr, m->indptr);
    cp(o->indices, m->indices);
    cp(o->slot_on, m->slot_on);
    cp(o->slot_no, m->slot_no);
    cp(o->diag_slot, m->diag_slot);
    cp(o->face_color, m->face_color);
    cp(o->cell_color, m->cell_color);
    cp(o->level_natural, m->level_natural);
    return KCFD_OK;
}

void kcfd_mesh_free(kcfd_host_mesh* m) { delete m; }

int kcfd_version(void) { return 100; }

int kcfd_last_error(char* buf, int32_t len) {
    if (!buf || len <= 0) return KCFD_BAD_INPUT;
    const std::string& e = kcfd::last_error();
    size_t k = std::min<size_t>(e.size(), (size_t)len - 1);
    std::memcpy(buf, e.data(), k);
    buf[k] = 0;
    return KCFD_OK;
}

}  // extern "C"
