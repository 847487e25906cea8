// mesh_build.cu -- connectivity and colouring of tri / quad / tet / hex meshes on the GPU.
//
// Produces, bit for bit, the layout the reference's MeshTetGPU::init / MeshTriGPU::init build
// (mesh/MeshTetGPU.cu:35-42, mesh/MeshTriGPU.cu:37-50):
//   * boundary faces of a tet mesh: every tet face rotated smallest-index-first
//     (mesh/MeshGPUCommon.cu:1371-1410), sorted lexicographically, faces meeting their
//     opposite-oriented twin removed (k_markDuplicateTris, :56-74);
//   * vertex order [free surface by colour | feature surface by colour | inner by colour]
//     through stable partitions and stable colour sorts (mesh/MeshTetGPU.cu:241-295,
//     mesh/MeshTriGPU.cu:597-671), elements remapped after each step;
//   * halfedge CSR with boundary dummies, CCW fan order, opposite and next
//     (mesh/MeshTriGPU.cu:128-214, mesh/MeshGPUCommon.cu:96-135,211-285,565-620); quad meshes
//     the same with faces of four corners (mesh/MeshQuadGPU.cu), the fan walk stepping to the
//     corner two after the target (getThirdVertex, mesh/MeshGPUCommon.cu:149-162) and the
//     colouring adjacency holding both diagonals (:1067-1097);
//   * halfface CSR, rows in tetrahedron order (mesh/MeshTetGPU.cu:113-142); for hex meshes the
//     boundary quads (mesh/MeshHexGPU.cu:141-164), the all-pairs colouring graph of a hexahedron
//     and the halfhex CSR (mesh/MeshHexGPU.cu:116-139, mesh/MeshGPUCommon.cu:1334-1368);
//   * boundary / feature flags (dihedral > 20 deg, mesh/MeshGPUCommon.cu:466-495) and face /
//     vertex normals (:363-434).
// Sorting uses the stable LSD radix sort of prim.cu. Colouring runs the reference's JPL round
// rule (mesh/VertexColoring.cu:76-105): by default with seeded hash priorities, each vertex
// taking the smallest colour none of its higher-priority neighbours has (the greedy colouring in
// priority order, computed round by round); with VSDMO_COLOR_ROUNDS in the seed the colour is the
// round (the reference's rule) with the hashed priorities of the seed's other bits; with
// VSDMO_COLOR_REFERENCE the colour is the round and the priorities are the reference's own n - i
// (VertexColoring.cu:107-125).
#include "vsdmo_internal.cuh"
#include <climits>
#include <cmath>

namespace vsdmo {
namespace {

enum BuildErr { BE_OK = 0, BE_INDEX = 1, BE_NAN = 2, BE_DEGENERATE = 3, BE_NONMANIFOLD = 4,
                BE_FAN = 5, BE_FEATURE_START = 6 };

// n: the number of vertices coloured together (i is local to them)
__device__ __forceinline__ uint32_t priority(uint32_t i, uint32_t seed, uint32_t n) {
    if (seed == VSDMO_COLOR_REFERENCE) return n - i;
    seed &= ~VSDMO_COLOR_ROUNDS;
    uint32_t h = i + seed * 0x9E3779B9u;
    h ^= h >> 16; h *= 0x85EBCA6Bu;
    h ^= h >> 13; h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

// the halfedge fans are walked by one thread per vertex in time quadratic in the fan's length
// (k_ccw, like the reference's k_sortCCWDummyOpposite): longer fans are refused
[[noreturn]] void throw_long_fan() {
    throw Error(VSDMO_E_VALENCE, "a vertex has more than " + std::to_string(SHORT_ROW_MAX) + " halfedges");
}

#define GRID_STRIDE(i, n) for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long)gridDim.x * blockDim.x)
constexpr unsigned FULL = 0xffffffffu;

__global__ void k_count_keys_u32(const uint32_t* keys, long n, int* counts) { GRID_STRIDE(i, n) atomicAdd(&counts[keys[i]], 1); }

__global__ void k_input(const float* xyz, int nV, const int* elems, long nIdx, float4* pos, int* err, int* nonzero_z) {
    GRID_STRIDE(i, nV) {
        float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        if (!isfinite(x) || !isfinite(y) || !isfinite(z)) atomicMax(err, BE_NAN);
        if (z != 0.f) *nonzero_z = 1;
        pos[i] = make_float4(x, y, z, 0.f);
    }
    GRID_STRIDE(i, nIdx) {
        int v = elems[i];
        if (v < 0 || v >= nV) atomicMax(err, BE_INDEX);
    }
}

__global__ void k_iota(uint32_t* a, long n) { GRID_STRIDE(i, n) a[i] = (uint32_t)i; }

template <class T>
__global__ void k_gather(const T* src, const uint32_t* idx, T* dst, long n) { GRID_STRIDE(i, n) dst[i] = src[idx[i]]; }

__global__ void k_gather_key(const uint32_t* src, const uint32_t* idx, uint32_t* dst, long n) {
    GRID_STRIDE(i, n) dst[i] = src[idx[i]];
}

// ---- tetrahedral boundary ---------------------------------------------------------------
__device__ __forceinline__ void smallest_first(int a, int b, int c, uint32_t* o) {
    if (a < b && a < c) { o[0] = a; o[1] = b; o[2] = c; }
    else if (b < a && b < c) { o[0] = b; o[1] = c; o[2] = a; }
    else { o[0] = c; o[1] = a; o[2] = b; }
}

__global__ void k_tet_faces(const int* tets, int nT, uint32_t* f0, uint32_t* f1, uint32_t* f2) {
    GRID_STRIDE(t, nT) {
        const int* v = tets + 4 * t;
        uint32_t o[3];
        smallest_first(v[2], v[1], v[0], o); f0[4 * t] = o[0]; f1[4 * t] = o[1]; f2[4 * t] = o[2];
        smallest_first(v[0], v[1], v[3], o); f0[4 * t + 1] = o[0]; f1[4 * t + 1] = o[1]; f2[4 * t + 1] = o[2];
        smallest_first(v[1], v[2], v[3], o); f0[4 * t + 2] = o[0]; f1[4 * t + 2] = o[1]; f2[4 * t + 2] = o[2];
        smallest_first(v[0], v[3], v[2], o); f0[4 * t + 3] = o[0]; f1[4 * t + 3] = o[1]; f2[4 * t + 3] = o[2];
    }
}

// faces bucketed by their first vertex: row f0 holds (f1 << 32 | f2) of every face (f0, f1, f2)
__global__ void k_face_bucket(const uint32_t* f0, const uint32_t* f1, const uint32_t* f2, long nF, int* cursor,
                              unsigned long long* out) {
    GRID_STRIDE(i, nF) out[atomicAdd(&cursor[f0[i]], 1)] = ((unsigned long long)f1[i] << 32) | f2[i];
}

// one warp per row a (grid-stride over rows): face (a, b, c) is a boundary face unless the row
// also holds its twin (a, c, b) (k_markDuplicateTris, mesh/MeshGPUCommon.cu:56-74); an exact
// repeat is a non-manifold input. The boundary faces get their place among the row's boundary
// faces in (b, c) order, so rows in vertex order give the lexicographic order of a sort.
__global__ void k_face_rows(const int* rs, const unsigned long long* fb, long K, uint8_t* bnd, int* rank, int* u,
                            int* err) {
    const int lane = threadIdx.x & 31;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < K; r += nw) {
        const int b0 = rs[r], n = rs[r + 1] - b0;
        for (int i = lane; i < n; i += 32) {
            const unsigned long long x = fb[b0 + i], twin = (x << 32) | (x >> 32);
            bool paired = false, repeat = false;
            for (int j = 0; j < n; ++j) {
                if (j == i) continue;
                const unsigned long long y = fb[b0 + j];
                repeat |= y == x;
                paired |= y == twin;
            }
            if (repeat) atomicMax(err, BE_NONMANIFOLD);
            bnd[b0 + i] = paired ? 0 : 1;
        }
        __syncwarp();
        int cnt = 0;
        for (int i = lane; i < n; i += 32) {
            if (!bnd[b0 + i]) continue;
            const unsigned long long x = fb[b0 + i];
            int k = 0;
            for (int j = 0; j < n; ++j) k += (bnd[b0 + j] && fb[b0 + j] < x) ? 1 : 0;
            rank[b0 + i] = k;
            ++cnt;
        }
        cnt = __reduce_add_sync(FULL, cnt);
        if (lane == 0) u[r] = cnt;
        __syncwarp();
    }
}

// one warp per row: the row's boundary faces to tris[offs[a] + rank], their vertices flagged
__global__ void k_face_emit(const int* rs, const unsigned long long* fb, const uint8_t* bnd, const int* rank,
                            const int* offs, long K, int* tris, uint8_t* isB2) {
    const int lane = threadIdx.x & 31;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < K; r += nw) {
        const int b0 = rs[r], n = rs[r + 1] - b0;
        for (int i = lane; i < n; i += 32) {
            if (!bnd[b0 + i]) continue;
            const long p = offs[r] + rank[b0 + i];
            const unsigned long long x = fb[b0 + i];
            const int b = (int)(x >> 32), c = (int)(x & 0xffffffffu);
            tris[3 * p] = (int)r; tris[3 * p + 1] = b; tris[3 * p + 2] = c;
            isB2[r] = 1; isB2[b] = 1; isB2[c] = 1;
        }
    }
}

// ---- hexahedral boundary (MeshHexGPU::initBoundary2D, mesh/MeshHexGPU.cu:141-164) --------------
// getQuadSmallestFirst: rotate so that the smallest index comes first (mesh/MeshGPUCommon.cu:37-54)
__device__ __forceinline__ void quad_smallest_first(int a, int b, int c, int d, uint32_t* o) {
    if (b < a && b < c && b < d) { o[0] = b; o[1] = c; o[2] = d; o[3] = a; }
    else if (c < a && c < b && c < d) { o[0] = c; o[1] = d; o[2] = a; o[3] = b; }
    else if (d < a && d < b && d < c) { o[0] = d; o[1] = a; o[2] = b; o[3] = c; }
    else { o[0] = a; o[1] = b; o[2] = c; o[3] = d; }
}

// the six faces of a hexahedron (k_constructQuadsFromHexahedra, mesh/MeshGPUCommon.cu:1412-1430)
__global__ void k_hex_faces(const int* hexes, int nH, uint32_t* f0, uint32_t* f1, uint32_t* f2, uint32_t* f3) {
    const int F[6][4] = { {0, 1, 2, 3}, {1, 5, 6, 2}, {3, 2, 6, 7}, {4, 0, 3, 7}, {1, 0, 4, 5}, {5, 4, 7, 6} };
    GRID_STRIDE(t, nH) {
        const int* v = hexes + 8 * t;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            uint32_t o[4];
            quad_smallest_first(v[F[f][0]], v[F[f][1]], v[F[f][2]], v[F[f][3]], o);
            f0[6 * t + f] = o[0]; f1[6 * t + f] = o[1]; f2[6 * t + f] = o[2]; f3[6 * t + f] = o[3];
        }
    }
}

__device__ __forceinline__ int cmp4(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1,
                                    uint32_t b2, uint32_t b3) {
    if (a0 != b0) return a0 < b0 ? -1 : 1;
    if (a1 != b1) return a1 < b1 ? -1 : 1;
    if (a2 != b2) return a2 < b2 ? -1 : 1;
    if (a3 != b3) return a3 < b3 ? -1 : 1;
    return 0;
}

// quads sorted lexicographically: (a,b,c,d) with b<d pairs with (a,d,c,b) (k_markDuplicateQuads)
__global__ void k_pair_quads(const uint32_t* s0, const uint32_t* s1, const uint32_t* s2, const uint32_t* s3, long nF,
                             uint8_t* paired, int* err) {
    GRID_STRIDE(i, nF) {
        const uint32_t a = s0[i], b = s1[i], c = s2[i], d = s3[i];
        if (i + 1 < nF && s0[i + 1] == a && s1[i + 1] == b && s2[i + 1] == c && s3[i + 1] == d) atomicMax(err, BE_NONMANIFOLD);
        if (b < d) {
            long lo = i + 1, hi = nF;
            while (lo < hi) {
                const long mid = (lo + hi) >> 1;
                if (cmp4(s0[mid], s1[mid], s2[mid], s3[mid], a, d, c, b) < 0) lo = mid + 1; else hi = mid;
            }
            if (lo < nF && s0[lo] == a && s1[lo] == d && s2[lo] == c && s3[lo] == b) { paired[i] = 1; paired[lo] = 1; }
        }
    }
}

__global__ void k_emit_boundary_quads(const int* idx, int nB, const uint32_t* s0, const uint32_t* s1, const uint32_t* s2,
                                      const uint32_t* s3, int* quads, uint8_t* isB2) {
    GRID_STRIDE(i, nB) {
        const int j = idx[i];
        const int a = s0[j], b = s1[j], c = s2[j], d = s3[j];
        quads[4 * i] = a; quads[4 * i + 1] = b; quads[4 * i + 2] = c; quads[4 * i + 3] = d;
        isB2[a] = 1; isB2[b] = 1; isB2[c] = 1; isB2[d] = 1;
    }
}

// every vertex pair of a hexahedron within [lo, lo+num) (mesh/MeshGPUCommon.cu:936-1037)
__global__ void k_hex_pairs(const int* hexes, int nH, int lo, int num, uint32_t* ks, uint32_t* vs, int* counter) {
    GRID_STRIDE(t, nH) {
        const int* v = hexes + 8 * t;
        for (int i = 0; i < 7; ++i)
            for (int j = i + 1; j < 8; ++j) {
                const int a = v[i] - lo, b = v[j] - lo;
                if (a >= 0 && a < num && b >= 0 && b < num) {
                    const int p = atomicAdd(counter, 2);
                    ks[p] = a; vs[p] = b; ks[p + 1] = b; vs[p + 1] = a;
                }
            }
    }
}

// halfhex of corner j: the other seven corners (k_constructHalfhexesNew, mesh/MeshGPUCommon.cu:1334-1368),
// two int4 per halfhex (the eighth value is -1)
__global__ void k_halfhexes(const uint32_t* order, long nHH, const int* hexes, int4* hh) {
    const int H[8][7] = { {1, 2, 3, 4, 5, 6, 7}, {5, 6, 2, 0, 4, 7, 3}, {6, 7, 3, 1, 5, 4, 0}, {7, 4, 0, 2, 6, 5, 1},
                          {0, 3, 7, 5, 1, 2, 6}, {4, 7, 6, 1, 0, 3, 2}, {5, 4, 7, 2, 1, 0, 3}, {6, 5, 4, 3, 2, 1, 0} };
    GRID_STRIDE(i, nHH) {
        const int e = (int)order[i], t = e >> 3, j = e & 7;
        const int* v = hexes + 8L * t;
        hh[2 * i] = make_int4(v[H[j][0]], v[H[j][1]], v[H[j][2]], v[H[j][3]]);
        hh[2 * i + 1] = make_int4(v[H[j][4]], v[H[j][5]], v[H[j][6]], -1);
    }
}

__global__ void k_not(const uint8_t* f, uint8_t* o, long n) { GRID_STRIDE(i, n) o[i] = f[i] ? 0 : 1; }

// ---- permutations -----------------------------------------------------------------------
// full-size maps from a range order: new_of_old / old_of_new are identity outside [start, start+num)
__global__ void k_range_maps(const int* order_local, int start, int num, int nTot, int* old_of_new, int* new_of_old) {
    GRID_STRIDE(i, nTot) {
        if (i < start || i >= start + num) { old_of_new[i] = (int)i; new_of_old[i] = (int)i; }
    }
    GRID_STRIDE(i, num) {
        int o = start + order_local[i];
        old_of_new[start + i] = o;
        new_of_old[o] = start + (int)i;
    }
}

__global__ void k_permute_verts(const int* old_of_new, int nTot, const float4* pin, float4* pout, const int* oin, int* oout) {
    GRID_STRIDE(i, nTot) {
        int o = old_of_new[i];
        pout[i] = pin[o];
        oout[i] = oin[o];
    }
}

__global__ void k_permute_u8(const int* old_of_new, int n, const uint8_t* in, uint8_t* out) {
    GRID_STRIDE(i, n) out[i] = in[old_of_new[i]];
}

__global__ void k_remap(int* idx, long n, const int* new_of_old, int limit) {
    GRID_STRIDE(i, n) {
        int v = idx[i];
        if (v >= 0 && v < limit) idx[i] = new_of_old[v];
    }
}

// ---- adjacency pairs ---------------------------------------------------------------------
__global__ void k_tet_edge_pairs(const int* tets, int nT, int lo, int num, uint32_t* ks, uint32_t* vs, int* counter) {
    const int E[6][2] = { {0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3} };
    GRID_STRIDE(t, nT) {
        const int* v = tets + 4 * t;
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            int a = v[E[e][0]] - lo, b = v[E[e][1]] - lo;
            if (a >= 0 && a < num && b >= 0 && b < num) {
                int p = atomicAdd(counter, 2);
                ks[p] = a; vs[p] = b; ks[p + 1] = b; vs[p + 1] = a;
            }
        }
    }
}

__global__ void k_tri_edge_pairs(const int* tris, int nTris, int lo, int num, uint32_t* ks, uint32_t* vs, int* counter) {
    const int E[3][2] = { {0, 1}, {0, 2}, {1, 2} };
    GRID_STRIDE(t, nTris) {
        const int* v = tris + 3 * t;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            int a = v[E[e][0]] - lo, b = v[E[e][1]] - lo;
            if (a >= 0 && a < num && b >= 0 && b < num) {
                int p = atomicAdd(counter, 2);
                ks[p] = a; vs[p] = b; ks[p + 1] = b; vs[p + 1] = a;
            }
        }
    }
}

// quad edges and both diagonals
__global__ void k_quad_edge_pairs(const int* quads, int nQ, int lo, int num, uint32_t* ks, uint32_t* vs, int* counter) {
    const int E[6][2] = { {0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 2}, {1, 3} };
    GRID_STRIDE(t, nQ) {
        const int* v = quads + 4 * t;
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            int a = v[E[e][0]] - lo, b = v[E[e][1]] - lo;
            if (a >= 0 && a < num && b >= 0 && b < num) {
                int p = atomicAdd(counter, 2);
                ks[p] = a; vs[p] = b; ks[p + 1] = b; vs[p + 1] = a;
            }
        }
    }
}

// ---- JPL colouring ---------------------------------------------------------------------------
__global__ void k_fill_int(int* a, long n, int v) { GRID_STRIDE(i, n) a[i] = v; }

// One JPL round c: an uncoloured vertex is coloured iff its priority beats every neighbour that
// is uncoloured or coloured in this round (rnd: the round each vertex was coloured in, -1 before).
// Its colour is c (round colours), or with first_fit the smallest colour none of its coloured
// neighbours has: those all have higher priorities and earlier rounds (two neighbours are never
// coloured in the same round), so the colours are the greedy colouring in priority order.
// prev: the previous round's count of uncoloured vertices in the same host read (null for the
// first round of one); when it is 0 every vertex has its colour and the round has nothing to do.
// maxc collects the largest first-fit colour.
__global__ void k_jpl_round(int n, const int* rowptr, const int* col, uint32_t seed, int c, int first_fit, int* colors,
                            int* rnd, int* remaining, const int* prev, int* maxc) {
    if (prev && *prev == 0) return;
    GRID_STRIDE(i, n) {
        if (rnd[i] != -1) continue;
        const uint32_t pi = priority((uint32_t)i, seed, (uint32_t)n);
        bool f = true;
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            const int j = col[e];
            const int jr = rnd[j];
            if ((jr != -1 && jr != c) || (int)i == j) continue;
            if (pi <= priority((uint32_t)j, seed, (uint32_t)n)) { f = false; break; }
        }
        if (!f) {
            atomicAdd(remaining, 1);
            continue;
        }
        int colour = c;
        if (first_fit) {
            // smallest colour not taken by a neighbour coloured in an earlier round
            unsigned long long used = 0ull;
            for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
                const int j = col[e];
                const int jr = rnd[j];
                if (jr == -1 || jr == c || (int)i == j) continue;
                const int cj = colors[j];
                if (cj < 64) used |= 1ull << cj;
            }
            if (~used) {
                colour = __ffsll((long long)~used) - 1;
            } else {
                for (colour = 64;; ++colour) {
                    bool taken = false;
                    for (int e = rowptr[i]; e < rowptr[i + 1] && !taken; ++e) {
                        const int j = col[e];
                        const int jr = rnd[j];
                        taken = jr != -1 && jr != c && (int)i != j && colors[j] == colour;
                    }
                    if (!taken) break;
                }
            }
            atomicMax(maxc, colour);
        }
        colors[i] = colour;
        rnd[i] = c;
    }
}

__global__ void k_add_const(int* a, long n, int v) { GRID_STRIDE(i, n) a[i] += v; }

// ---- surface ------------------------------------------------------------------------------------
// face normal from corners 0, 1 and 2 (triangles) or 0, 1 and 3 (quads)
__global__ void k_face_normals(const int* tris, int fk, int nTris, const float4* pos, float* fn, int* err) {
    GRID_STRIDE(t, nTris) {
        const int* f = tris + (long)fk * t;
        float4 p0 = pos[f[0]], p1 = pos[f[1]], p2 = pos[f[fk == 4 ? 3 : 2]];
        float e0x = p1.x - p0.x, e0y = p1.y - p0.y, e0z = p1.z - p0.z;
        float e1x = p2.x - p0.x, e1y = p2.y - p0.y, e1z = p2.z - p0.z;
        if (err) {
            float l0 = sqrtf(e0x * e0x + e0y * e0y + e0z * e0z);
            float l1 = sqrtf(e1x * e1x + e1y * e1y + e1z * e1z);
            if (l0 < 1e-6f || l1 < 1e-6f) atomicMax(err, BE_DEGENERATE);
        }
        float nx = e0y * e1z - e0z * e1y, ny = e0z * e1x - e0x * e1z, nz = e0x * e1y - e0y * e1x;
        float len = sqrtf(nx * nx + ny * ny + nz * nz);
        fn[3 * t] = nx / len; fn[3 * t + 1] = ny / len; fn[3 * t + 2] = nz / len;
    }
}

// first-pass halfedges from the sorted (src, fk*t+j) pairs
__global__ void k_he_records(const uint32_t* order, long nHE, const int* tris, int fk, int4* he) {
    GRID_STRIDE(i, nHE) {
        int e = (int)order[i], t = e / fk, j = e % fk;
        he[i] = make_int4(tris[(long)fk * t + (j + 1) % fk], -1, t, 0);
    }
}

// opposite = last halfedge of the target's row that points back to the source
__global__ void k_opposite(const uint32_t* srcs, int4* he, long nHE, const int* rowptr) {
    GRID_STRIDE(i, nHE) {
        int src = (int)srcs[i], dst = he[i].x, opp = -1;
        for (int q = rowptr[dst]; q < rowptr[dst + 1]; ++q) if (he[q].x == src) opp = q;
        he[i].y = opp;
    }
}

__global__ void k_flags_b1_feat(const uint32_t* srcs, const int4* he, long nHE, const float* fn, uint8_t* isB1,
                                uint8_t* isFeat, int flat) {
    GRID_STRIDE(i, nHE) {
        int src = (int)srcs[i];
        int4 h = he[i];
        if (h.y == -1) {
            isB1[src] = 1;
            if (!flat) { isFeat[src] = 1; isFeat[h.x] = 1; }
            continue;
        }
        if (flat) continue;
        const float* f1 = fn + 3 * (long)h.z;
        const float* f2 = fn + 3 * (long)he[h.y].z;
        float dot = f1[0] * f2[0] + f1[1] * f2[1] + f1[2] * f2[2];
        float len = sqrtf((f1[0] * f1[0] + f1[1] * f1[1] + f1[2] * f1[2]) * (f2[0] * f2[0] + f2[1] * f2[1] + f2[2] * f2[2]));
        // the reference keeps the angle as a float (float angle = 180.f / M_PI * acosf(..),
        // MeshGPUCommon.cu:485-488): the double product is rounded before the compare
        const float angle = (float)(180.0 / 3.14159265358979323846 * (double)acosf(dot / len));
        if (angle > 20.f) { isFeat[src] = 1; isFeat[h.x] = 1; }
    }
}

__global__ void k_copy_u8(const uint8_t* a, uint8_t* b, long n) { GRID_STRIDE(i, n) b[i] = a[i]; }

__global__ void k_dummy_flags(const int4* he, long n, uint8_t* f) { GRID_STRIDE(i, n) f[i] = he[i].y == -1 ? 1 : 0; }

// real halfedges (sorted) followed by the dummies in the sorted order of their twins
__global__ void k_with_dummies(const uint32_t* srcs, const int4* he, long nHE1, const int* didx, int nD,
                               uint32_t* keys, int4* rec) {
    GRID_STRIDE(i, nHE1) { keys[i] = srcs[i]; rec[i] = make_int4(he[i].x, -1, he[i].z, 0); }
    GRID_STRIDE(j, nD) {
        int i = didx[j];
        keys[nHE1 + j] = (uint32_t)he[i].x;
        rec[nHE1 + j] = make_int4((int)srcs[i], -1, -1, 0);
    }
}

__device__ __forceinline__ int third_vertex(const int* t, int src, int dst) {
    if (t[0] != src && t[0] != dst) return t[0];
    if (t[1] != src && t[1] != dst) return t[1];
    return t[2];
}

// the corner two after dst (getThirdVertex for quads)
__device__ __forceinline__ int third_vertex_quad(const int* q, int dst) {
    if (dst == q[1]) return q[3];
    if (dst == q[2]) return q[0];
    if (dst == q[3]) return q[1];
    return q[2];
}

__global__ void k_ccw(int nS, const int* rowptr, const int4* in, int4* out, const uint8_t* isB1, const uint8_t* isFeat,
                      const int* tris, int fk, int* err) {
    GRID_STRIDE(src, nS) {
        const int start = rowptr[src], n = rowptr[src + 1] - start;
        if (n == 0) { atomicMax(err, BE_FAN); continue; }
        int outPos = 0;
        int4 h = in[start];
        bool bad = false;
        if (isB1[src]) {
            int j = 0;
            while (true) {
                if (h.y < 0) { bad = true; break; }
                if (in[h.y].z == -1) break;
                if (++j == n) { bad = true; break; }
                h = in[start + j];
            }
        } else if (isFeat[src]) {
            h.x = INT_MAX;
            for (int j = 0; j < n; ++j) {
                int4 t = in[start + j];
                if (isFeat[t.x] && t.x < h.x) h = t;
            }
            if (h.x == INT_MAX) { atomicMax(err, BE_FEATURE_START); continue; }
        } else {
            for (int i = 1; i < n; ++i) { int4 t = in[start + i]; if (t.x < h.x) h = t; }
        }
        if (bad) { atomicMax(err, BE_FAN); continue; }
        out[start + outPos++] = h;
        bool found;
        do {
            int currDst = h.x, currTri = h.z;
            if (currTri == -1) { bad = true; break; }
            int nextVert = fk == 4 ? third_vertex_quad(tris + 4 * (long)currTri, currDst)
                                   : third_vertex(tris + 3 * (long)currTri, (int)src, currDst);
            found = false;
            for (int j = 0; j < n; ++j) {
                int4 t = in[start + j];
                if (t.x == nextVert) {
                    if (outPos >= n) { bad = true; break; }
                    found = true; h = t; out[start + outPos++] = h;
                }
            }
            if (bad) break;
        } while (found && outPos < n);
        if (bad || outPos != n) atomicMax(err, BE_FAN);
    }
}

__global__ void k_opp_next(int nS, const int* rowptr, int4* he) {
    GRID_STRIDE(v, nS) {
        for (int i = rowptr[v]; i < rowptr[v + 1]; ++i) {
            int4 h = he[i];
            int opp = -1, nxt = h.w;
            for (int q = rowptr[h.x]; q < rowptr[h.x + 1]; ++q) {
                int4 o = he[q];
                if (o.x == (int)v) opp = q;
                if (o.z == h.z) nxt = q;
            }
            he[i].y = opp; he[i].w = nxt;
        }
    }
}

__global__ void k_max_row(const int* rowptr, int n, int* mx) {
    GRID_STRIDE(i, n) atomicMax(mx, rowptr[i + 1] - rowptr[i]);
}

__global__ void k_vertex_normals(int nS, const int* rowptr, const int4* he, const float* fn, float* vn) {
    GRID_STRIDE(v, nS) {
        float nx = 0.f, ny = 0.f, nz = 0.f;
        for (int i = rowptr[v]; i < rowptr[v + 1]; ++i) {
            int f = he[i].z;
            if (f != -1) { nx += fn[3 * f]; ny += fn[3 * f + 1]; nz += fn[3 * f + 2]; }
        }
        float len = sqrtf(nx * nx + ny * ny + nz * nz);
        vn[3 * v] = nx / len; vn[3 * v + 1] = ny / len; vn[3 * v + 2] = nz / len;
    }
}

// ---- halffaces ------------------------------------------------------------------------------------
__global__ void k_halffaces(const uint32_t* order, long nH, const int* tets, int4* hf) {
    GRID_STRIDE(i, nH) {
        int e = (int)order[i], t = e >> 2, j = e & 3;
        const int* v = tets + 4 * (long)t;
        int4 o;
        if (j == 0) o = make_int4(v[1], v[2], v[3], t);
        else if (j == 1) o = make_int4(v[0], v[3], v[2], t);
        else if (j == 2) o = make_int4(v[0], v[1], v[3], t);
        else o = make_int4(v[0], v[2], v[1], t);
        hf[i] = o;
    }
}

__global__ void k_final_perm(const int* orig_of_cur, int nV, int* new_of_old) {
    GRID_STRIDE(i, nV) new_of_old[orig_of_cur[i]] = (int)i;
}

inline int G(long n) { return grid_for(n, 256); }

void check_err(const DBuf<int>& err, cudaStream_t s, const char* stage) {
    int e = read_scalar(err.p, s);
    switch (e) {
    case BE_OK: return;
    case BE_INDEX: throw Error(VSDMO_E_ARG, std::string(stage) + ": element index out of range");
    case BE_NAN: throw Error(VSDMO_E_NAN, std::string(stage) + ": non-finite vertex coordinate");
    case BE_DEGENERATE: throw Error(VSDMO_E_ARG, std::string(stage) + ": degenerate triangle (edge shorter than 1e-6)");
    case BE_NONMANIFOLD: throw Error(VSDMO_E_NONMANIFOLD, std::string(stage) + ": a face occurs twice with the same orientation");
    case BE_FAN: throw Error(VSDMO_E_NONMANIFOLD, std::string(stage) + ": a vertex fan is open or non-manifold");
    case BE_FEATURE_START: throw Error(VSDMO_E_NONMANIFOLD, std::string(stage) + ": feature vertex without feature neighbour");
    default: throw Error(VSDMO_E_CUDA, std::string(stage) + ": unknown build error");
    }
}

// Shared state of one build.
struct Builder {
    Mesh& m;
    cudaStream_t s;
    DBuf<int> orig_of_cur;
    DBuf<int> err;
    explicit Builder(Mesh& mm) : m(mm), s(mm.stream) {}

    // apply a permutation of range [start, start+num) given as order_local (new -> old, local)
    void permute_range(const int* order_local, int start, int num, std::vector<DBuf<uint8_t>*> flags,
                       std::vector<std::pair<int*, long>> elem_arrays, int remap_limit) {
        const int nTot = m.nV;
        DBuf<int> oon(nTot, s), noo(nTot, s);
        k_range_maps<<<G(nTot), 256, 0, s>>>(order_local, start, num, nTot, oon.p, noo.p);
        VSDMO_CHECK_LAUNCH();
        DBuf<float4> p2(nTot, s);
        DBuf<int> o2(nTot, s);
        k_permute_verts<<<G(nTot), 256, 0, s>>>(oon.p, nTot, m.pos.p, p2.p, orig_of_cur.p, o2.p);
        VSDMO_CHECK_LAUNCH();
        m.pos = std::move(p2);
        orig_of_cur = std::move(o2);
        for (DBuf<uint8_t>* f : flags) {
            if (!f->p) continue;
            long n = (long)f->n;
            DBuf<uint8_t> f2(n, s);
            k_permute_u8<<<G(n), 256, 0, s>>>(oon.p, (int)n, f->p, f2.p);
            VSDMO_CHECK_LAUNCH();
            *f = std::move(f2);
        }
        for (auto& ea : elem_arrays) {
            if (!ea.first || ea.second == 0) continue;
            k_remap<<<G(ea.second), 256, 0, s>>>(ea.first, ea.second, noo.p, remap_limit);
            VSDMO_CHECK_LAUNCH();
        }
    }

    // stable partition of [0, n): flag == first_value first; returns the number of those
    int stable_partition(const uint8_t* d_flags, int n, int first_value, DBuf<int>& order) {
        order.alloc(n, s);
        return stable_partition_flags(d_flags, n, first_value, order.p, s);
    }

    // colour the range [lo, lo+num) given its adjacency pairs; sort it by colour
    int color_range(int lo, int num, DBuf<uint32_t>& ks, DBuf<uint32_t>& vs, int npairs, std::vector<int>& offs_host,
                    DBuf<int>& offs_dev, std::vector<DBuf<uint8_t>*> flags, std::vector<std::pair<int*, long>> elems) {
        // adjacency CSR with sorted unique rows
        DBuf<int> rowptr(num + 1, s);
        DBuf<int> col;
        if (npairs > 0) {
            col.alloc(npairs, s);
            csr_unique_from_pairs(ks.p, vs.p, npairs, num, rowptr.p, col.p, s);
        } else {
            rowptr.zero();
            col.alloc(1, s);
        }
        // JPL rounds, CH per host read: round c leaves remaining[c % CH] uncoloured vertices; the
        // rounds after the last one find nobody uncoloured and change nothing; remaining[CH]
        // collects the largest first-fit colour
        constexpr int CH = 16;
        const int first_fit = m.seed != VSDMO_COLOR_REFERENCE && !(m.seed & VSDMO_COLOR_ROUNDS) ? 1 : 0;
        DBuf<int> colors(num, s), rnd(num, s), remaining(CH + 1, s);
        k_fill_int<<<G(num), 256, 0, s>>>(rnd.p, num, -1);
        VSDMO_CHECK_LAUNCH();
        remaining.zero();
        int nc = -1;
        std::vector<int> left;
        for (int c0 = 0; nc < 0; c0 += CH) {
            if (c0 > num + 1) throw Error(VSDMO_E_CUDA, "colouring did not terminate");
            VSDMO_CUDA(cudaMemsetAsync(remaining.p, 0, sizeof(int) * CH, s));
            for (int i = 0; i < CH; ++i) {
                k_jpl_round<<<G(num), 256, 0, s>>>(num, rowptr.p, col.p, m.seed, c0 + i, first_fit, colors.p, rnd.p,
                                                   remaining.p + i, i > 0 ? remaining.p + i - 1 : nullptr,
                                                   remaining.p + CH);
                VSDMO_CHECK_LAUNCH();
            }
            left = remaining.to_host();
            for (int i = 0; i < CH && nc < 0; ++i)
                if (left[i] == 0) nc = c0 + i + 1;
        }
        if (first_fit) nc = left[CH] + 1;
        // the colours are dense: every round colours the top-priority vertex left, and a
        // first-fit colour k has neighbours of every colour below k
        // stable sort of the range by colour
        DBuf<uint32_t> ck(num, s), order(num, s);
        VSDMO_CUDA(cudaMemcpyAsync(ck.p, colors.p, sizeof(int) * num, cudaMemcpyDeviceToDevice, s));
        k_iota<<<G(num), 256, 0, s>>>(order.p, num);
        VSDMO_CHECK_LAUNCH();
        radix_sort_pairs(ck.p, order.p, num, bits_for((uint32_t)(nc > 1 ? nc - 1 : 1)), s);
        offs_dev.alloc(nc + 1, s);
        rowptr_from_sorted(ck.p, num, nc, offs_dev.p, s);
        k_add_const<<<G(nc + 1), 256, 0, s>>>(offs_dev.p, nc + 1, lo);
        VSDMO_CHECK_LAUNCH();
        offs_host = offs_dev.to_host();
        permute_range((const int*)order.p, lo, num, flags, elems, m.nV);
        return nc;
    }

    void surface_init() {
        const int nS = m.nSurf;
        const long nHE1 = (long)m.fk * m.nTris;
        m.fn.alloc(3L * m.nTris, s);
        err.zero();
        k_face_normals<<<G(m.nTris), 256, 0, s>>>(m.tris.p, m.fk, m.nTris, m.pos.p, m.fn.p, err.p);
        VSDMO_CHECK_LAUNCH();
        check_err(err, s, "surface");
        // first-pass halfedges
        {
            DBuf<uint32_t> keys(nHE1, s), order(nHE1, s);
            VSDMO_CUDA(cudaMemcpyAsync(keys.p, m.tris.p, sizeof(int) * nHE1, cudaMemcpyDeviceToDevice, s));
            DBuf<int> rowptr(nS + 1, s);
            if (stable_sort_short_rows(keys.p, order.p, nHE1, nS, rowptr.p, s) > SHORT_ROW_MAX) throw_long_fan();
            DBuf<int4> he(nHE1, s);
            k_he_records<<<G(nHE1), 256, 0, s>>>(order.p, nHE1, m.tris.p, m.fk, he.p);
            VSDMO_CHECK_LAUNCH();
            k_opposite<<<G(nHE1), 256, 0, s>>>(keys.p, he.p, nHE1, rowptr.p);
            VSDMO_CHECK_LAUNCH();
            m.isB1.alloc(nS, s); m.isB1.zero();
            m.isFeat.alloc(nS, s); m.isFeat.zero();
            k_flags_b1_feat<<<G(nHE1), 256, 0, s>>>(keys.p, he.p, nHE1, m.fn.p, m.isB1.p, m.isFeat.p, m.isFlat);
            VSDMO_CHECK_LAUNCH();
            if (m.isFlat) {
                k_copy_u8<<<G(nS), 256, 0, s>>>(m.isB1.p, m.isFeat.p, nS);
                VSDMO_CHECK_LAUNCH();
            }
        }
        // free first, feature last
        {
            DBuf<int> order;
            int nFree = stable_partition(m.isFeat.p, nS, 0, order);
            std::vector<std::pair<int*, long>> el = { {m.tris.p, (long)m.fk * m.nTris} };
            if (m.type == VSDMO_TET || m.type == VSDMO_HEX) el.push_back({m.elems.p, (long)m.k * m.nE});
            permute_range(order.p, 0, nS, {&m.isB1, &m.isFeat}, el, nS);
            m.nFeature = nS - nFree;
        }
        const int nFree = nS - m.nFeature;
        for (int part = 0; part < 2; ++part) {
            const int lo = part == 0 ? 0 : nFree, num = part == 0 ? nFree : m.nFeature;
            std::vector<int>& oh = part == 0 ? m.col_free : m.col_feature;
            DBuf<int>& od = part == 0 ? m.d_col_free : m.d_col_feature;
            int& nc = part == 0 ? m.nColFree : m.nColFeature;
            if (num <= 0) {
                oh.assign(1, lo);
                od.alloc(1, s);
                VSDMO_CUDA(cudaMemcpyAsync(od.p, oh.data(), sizeof(int), cudaMemcpyHostToDevice, s));
                nc = 0;
                continue;
            }
            long cap = m.type == VSDMO_TET ? 12L * m.nE : m.type == VSDMO_HEX ? 56L * m.nE : (m.fk == 4 ? 12L : 6L) * m.nTris;
            DBuf<uint32_t> ks(cap, s), vs(cap, s);
            DBuf<int> cnt(1, s);
            cnt.zero();
            if (m.type == VSDMO_HEX)
                k_hex_pairs<<<G(m.nE), 256, 0, s>>>(m.elems.p, m.nE, lo, num, ks.p, vs.p, cnt.p);
            else if (m.type == VSDMO_TET)
                k_tet_edge_pairs<<<G(m.nE), 256, 0, s>>>(m.elems.p, m.nE, lo, num, ks.p, vs.p, cnt.p);
            else if (m.fk == 4)
                k_quad_edge_pairs<<<G(m.nTris), 256, 0, s>>>(m.tris.p, m.nTris, lo, num, ks.p, vs.p, cnt.p);
            else
                k_tri_edge_pairs<<<G(m.nTris), 256, 0, s>>>(m.tris.p, m.nTris, lo, num, ks.p, vs.p, cnt.p);
            VSDMO_CHECK_LAUNCH();
            int np = read_scalar(cnt.p, s);
            std::vector<std::pair<int*, long>> el = { {m.tris.p, (long)m.fk * m.nTris} };
            if (m.type == VSDMO_TET || m.type == VSDMO_HEX) el.push_back({m.elems.p, (long)m.k * m.nE});
            nc = color_range(lo, num, ks, vs, np, oh, od, {&m.isB1, &m.isFeat}, el);
        }
        final_halfedges();
        m.vn.alloc(3L * nS, s);
        k_vertex_normals<<<G(nS), 256, 0, s>>>(nS, m.he_rowptr.p, m.he.p, m.fn.p, m.vn.p);
        VSDMO_CHECK_LAUNCH();
    }

    void final_halfedges() {
        const int nS = m.nSurf;
        const long nHE1 = (long)m.fk * m.nTris;
        DBuf<uint32_t> keys(nHE1, s), order(nHE1, s);
        VSDMO_CUDA(cudaMemcpyAsync(keys.p, m.tris.p, sizeof(int) * nHE1, cudaMemcpyDeviceToDevice, s));
        DBuf<int> rowptr1(nS + 1, s);
        if (stable_sort_short_rows(keys.p, order.p, nHE1, nS, rowptr1.p, s) > SHORT_ROW_MAX) throw_long_fan();
        DBuf<int4> he1(nHE1, s);
        k_he_records<<<G(nHE1), 256, 0, s>>>(order.p, nHE1, m.tris.p, m.fk, he1.p);
        VSDMO_CHECK_LAUNCH();
        k_opposite<<<G(nHE1), 256, 0, s>>>(keys.p, he1.p, nHE1, rowptr1.p);
        VSDMO_CHECK_LAUNCH();
        DBuf<uint8_t> df(nHE1, s);
        k_dummy_flags<<<G(nHE1), 256, 0, s>>>(he1.p, nHE1, df.p);
        VSDMO_CHECK_LAUNCH();
        DBuf<int> didx(nHE1, s);
        const int nD = compact_flags(df.p, nHE1, didx.p, s);
        const long nHE = nHE1 + nD;
        DBuf<uint32_t> k2(nHE, s), o2(nHE, s);
        DBuf<int4> rec(nHE, s);
        k_with_dummies<<<G(nHE), 256, 0, s>>>(keys.p, he1.p, nHE1, didx.p, nD, k2.p, rec.p);
        VSDMO_CHECK_LAUNCH();
        m.he_rowptr.alloc(nS + 1, s);
        if (stable_sort_short_rows(k2.p, o2.p, nHE, nS, m.he_rowptr.p, s) > SHORT_ROW_MAX) throw_long_fan();
        DBuf<int4> in(nHE, s);
        k_gather<int4><<<G(nHE), 256, 0, s>>>(rec.p, o2.p, in.p, nHE);
        VSDMO_CHECK_LAUNCH();
        k_opposite<<<G(nHE), 256, 0, s>>>(k2.p, in.p, nHE, m.he_rowptr.p);
        VSDMO_CHECK_LAUNCH();
        m.he.alloc(nHE, s);
        err.zero();
        k_ccw<<<G(nS), 256, 0, s>>>(nS, m.he_rowptr.p, in.p, m.he.p, m.isB1.p, m.isFeat.p, m.tris.p, m.fk, err.p);
        VSDMO_CHECK_LAUNCH();
        check_err(err, s, "halfedges");
        k_opp_next<<<G(nS), 256, 0, s>>>(nS, m.he_rowptr.p, m.he.p);
        VSDMO_CHECK_LAUNCH();
        DBuf<int> mx(1, s);
        mx.zero();
        k_max_row<<<G(nS), 256, 0, s>>>(m.he_rowptr.p, nS, mx.p);
        VSDMO_CHECK_LAUNCH();
        m.maxHE = read_scalar(mx.p, s);
        m.nHE = (int)nHE;
    }

    void tet_boundary() {
        const int nT = m.nE, nV = m.nV;
        const long nF = 4L * nT;
        DBuf<uint32_t> f0(nF, s), f1(nF, s), f2(nF, s);
        k_tet_faces<<<G(nT), 256, 0, s>>>(m.elems.p, nT, f0.p, f1.p, f2.p);
        VSDMO_CHECK_LAUNCH();
        // bucket the faces by first vertex (counting sort), then pair each row's faces in place
        DBuf<int> counts(nV, s), rs((long)nV + 1, s), cursor(nV, s), u(nV, s), offs((long)nV + 1, s), rank(nF, s);
        DBuf<unsigned long long> fb(nF, s);
        DBuf<uint8_t> bnd(nF, s);
        counts.zero();
        k_count_keys_u32<<<G(nF), 256, 0, s>>>(f0.p, nF, counts.p);
        VSDMO_CHECK_LAUNCH();
        exclusive_scan(counts.p, rs.p, nV, rs.p + nV, s);
        if (longest_row(rs.p, nV, s) > SHORT_ROW_MAX)
            throw Error(VSDMO_E_VALENCE, "a vertex is the first corner of more than " + std::to_string(SHORT_ROW_MAX) +
                                             " tetrahedron faces (more than ~1365 tetrahedra around one vertex)");
        VSDMO_CUDA(cudaMemcpyAsync(cursor.p, rs.p, sizeof(int) * nV, cudaMemcpyDeviceToDevice, s));
        k_face_bucket<<<G(nF), 256, 0, s>>>(f0.p, f1.p, f2.p, nF, cursor.p, fb.p);
        VSDMO_CHECK_LAUNCH();
        err.zero();
        k_face_rows<<<G(32L * nV), 256, 0, s>>>(rs.p, fb.p, nV, bnd.p, rank.p, u.p, err.p);
        VSDMO_CHECK_LAUNCH();
        check_err(err, s, "boundary faces");
        exclusive_scan(u.p, offs.p, nV, offs.p + nV, s);
        const int nB = read_scalar(offs.p + nV, s);
        m.nTris = nB;
        m.tris.alloc(3L * nB, s);
        m.isB2.alloc(m.nV, s);
        m.isB2.zero();
        k_face_emit<<<G(32L * nV), 256, 0, s>>>(rs.p, fb.p, bnd.p, rank.p, offs.p, nV, m.tris.p, m.isB2.p);
        VSDMO_CHECK_LAUNCH();
    }

    void hex_boundary() {
        const int nH = m.nE;
        const long nF = 6L * nH;
        DBuf<uint32_t> f0(nF, s), f1(nF, s), f2(nF, s), f3(nF, s), key(nF, s), order(nF, s);
        k_hex_faces<<<G(nH), 256, 0, s>>>(m.elems.p, nH, f0.p, f1.p, f2.p, f3.p);
        VSDMO_CHECK_LAUNCH();
        k_iota<<<G(nF), 256, 0, s>>>(order.p, nF);
        VSDMO_CHECK_LAUNCH();
        const int bits = bits_for((uint32_t)(m.nV - 1));
        const uint32_t* comps[4] = { f3.p, f2.p, f1.p, f0.p };
        for (int c = 0; c < 4; ++c) {
            k_gather_key<<<G(nF), 256, 0, s>>>(comps[c], order.p, key.p, nF);
            VSDMO_CHECK_LAUNCH();
            radix_sort_pairs(key.p, order.p, nF, bits, s);
        }
        DBuf<uint32_t> s0(nF, s), s1(nF, s), s2(nF, s), s3(nF, s);
        k_gather_key<<<G(nF), 256, 0, s>>>(f0.p, order.p, s0.p, nF);
        k_gather_key<<<G(nF), 256, 0, s>>>(f1.p, order.p, s1.p, nF);
        k_gather_key<<<G(nF), 256, 0, s>>>(f2.p, order.p, s2.p, nF);
        k_gather_key<<<G(nF), 256, 0, s>>>(f3.p, order.p, s3.p, nF);
        VSDMO_CHECK_LAUNCH();
        DBuf<uint8_t> paired(nF, s), unpaired(nF, s);
        paired.zero();
        err.zero();
        k_pair_quads<<<G(nF), 256, 0, s>>>(s0.p, s1.p, s2.p, s3.p, nF, paired.p, err.p);
        VSDMO_CHECK_LAUNCH();
        check_err(err, s, "boundary faces");
        k_not<<<G(nF), 256, 0, s>>>(paired.p, unpaired.p, nF);
        VSDMO_CHECK_LAUNCH();
        DBuf<int> bidx(nF, s);
        const int nB = compact_flags(unpaired.p, nF, bidx.p, s);
        m.nTris = nB;
        m.tris.alloc(4L * nB, s);
        m.isB2.alloc(m.nV, s);
        m.isB2.zero();
        k_emit_boundary_quads<<<G(nB), 256, 0, s>>>(bidx.p, nB, s0.p, s1.p, s2.p, s3.p, m.tris.p, m.isB2.p);
        VSDMO_CHECK_LAUNCH();
    }

    void hex_halfhexes() {
        const long nHH = 8L * m.nE;
        DBuf<uint32_t> keys(nHH, s), order(nHH, s);
        VSDMO_CUDA(cudaMemcpyAsync(keys.p, m.elems.p, sizeof(int) * nHH, cudaMemcpyDeviceToDevice, s));
        k_iota<<<G(nHH), 256, 0, s>>>(order.p, nHH);
        VSDMO_CHECK_LAUNCH();
        radix_sort_pairs(keys.p, order.p, nHH, bits_for((uint32_t)(m.nV - 1)), s);
        m.hf_rowptr.alloc(m.nV + 1, s);
        rowptr_from_sorted(keys.p, nHH, m.nV, m.hf_rowptr.p, s);
        m.hh.alloc(2 * nHH, s);
        k_halfhexes<<<G(nHH), 256, 0, s>>>(order.p, nHH, m.elems.p, m.hh.p);
        VSDMO_CHECK_LAUNCH();
        DBuf<int> mx(1, s);
        mx.zero();
        k_max_row<<<G(m.nV), 256, 0, s>>>(m.hf_rowptr.p, m.nV, mx.p);
        VSDMO_CHECK_LAUNCH();
        m.maxTets = read_scalar(mx.p, s);
    }

    void tet_halffaces() {
        const long nH = 4L * m.nE;
        DBuf<uint32_t> keys(nH, s), order(nH, s);
        VSDMO_CUDA(cudaMemcpyAsync(keys.p, m.elems.p, sizeof(int) * nH, cudaMemcpyDeviceToDevice, s));
        m.hf_rowptr.alloc(m.nV + 1, s);
        stable_sort_short_rows(keys.p, order.p, nH, m.nV, m.hf_rowptr.p, s);
        m.hf.alloc(nH, s);
        k_halffaces<<<G(nH), 256, 0, s>>>(order.p, nH, m.elems.p, m.hf.p);
        VSDMO_CHECK_LAUNCH();
        DBuf<int> mx(1, s);
        mx.zero();
        k_max_row<<<G(m.nV), 256, 0, s>>>(m.hf_rowptr.p, m.nV, mx.p);
        VSDMO_CHECK_LAUNCH();
        m.maxTets = read_scalar(mx.p, s);
    }

    void run(const float* d_xyz, const int* d_elems) {
        const long nIdx = (long)m.nE * m.k;
        m.pos.alloc(m.nV, s);
        m.elems.alloc(nIdx, s);
        VSDMO_CUDA(cudaMemcpyAsync(m.elems.p, d_elems, sizeof(int) * nIdx, cudaMemcpyDeviceToDevice, s));
        err.alloc(1, s);
        err.zero();
        DBuf<int> nz(1, s);
        nz.zero();
        k_input<<<G(std::max<long>(m.nV, nIdx)), 256, 0, s>>>(d_xyz, m.nV, m.elems.p, nIdx, m.pos.p, err.p, nz.p);
        VSDMO_CHECK_LAUNCH();
        check_err(err, s, "input");
        orig_of_cur.alloc(m.nV, s);
        k_iota<<<G(m.nV), 256, 0, s>>>((uint32_t*)orig_of_cur.p, m.nV);
        VSDMO_CHECK_LAUNCH();
        if (m.type == VSDMO_TRI || m.type == VSDMO_QUAD) {
            m.fk = m.k;
            m.isFlat = read_scalar(nz.p, s) ? 0 : 1;
            m.nSurf = m.nV;
            m.nTris = m.nE;
            m.tris.alloc(nIdx, s);
            VSDMO_CUDA(cudaMemcpyAsync(m.tris.p, m.elems.p, sizeof(int) * nIdx, cudaMemcpyDeviceToDevice, s));
            m.col_inner.assign(1, m.nV);
            m.d_col_inner.alloc(1, s);
            VSDMO_CUDA(cudaMemcpyAsync(m.d_col_inner.p, m.col_inner.data(), sizeof(int), cudaMemcpyHostToDevice, s));
            surface_init();
            VSDMO_CUDA(cudaMemcpyAsync(m.elems.p, m.tris.p, sizeof(int) * nIdx, cudaMemcpyDeviceToDevice, s));
        } else if (m.type == VSDMO_TET) {
            m.fk = 3;
            m.isFlat = 0;
            tet_boundary();
            {
                DBuf<int> order;
                int nS = stable_partition(m.isB2.p, m.nV, 1, order);
                permute_range(order.p, 0, m.nV, {&m.isB2}, { {m.tris.p, 3L * m.nTris}, {m.elems.p, 4L * m.nE} }, m.nV);
                m.nSurf = nS;
            }
            const int nI = m.nV - m.nSurf;
            if (nI > 0) {
                DBuf<uint32_t> ks(12L * m.nE, s), vs(12L * m.nE, s);
                DBuf<int> cnt(1, s);
                cnt.zero();
                k_tet_edge_pairs<<<G(m.nE), 256, 0, s>>>(m.elems.p, m.nE, m.nSurf, nI, ks.p, vs.p, cnt.p);
                VSDMO_CHECK_LAUNCH();
                int np = read_scalar(cnt.p, s);
                m.nColInner = color_range(m.nSurf, nI, ks, vs, np, m.col_inner, m.d_col_inner, {&m.isB2},
                                          { {m.tris.p, 3L * m.nTris}, {m.elems.p, 4L * m.nE} });
            } else {
                m.nColInner = 0;
                m.col_inner.assign(1, m.nSurf);
                m.d_col_inner.alloc(1, s);
                VSDMO_CUDA(cudaMemcpyAsync(m.d_col_inner.p, m.col_inner.data(), sizeof(int), cudaMemcpyHostToDevice, s));
            }
            if (m.nSurf > 0) surface_init();
            tet_halffaces();
        } else {  // VSDMO_HEX (MeshHexGPU::init, mesh/MeshHexGPU.cu:35-43)
            m.fk = 4;
            m.isFlat = 0;
            hex_boundary();
            {
                DBuf<int> order;
                int nS = stable_partition(m.isB2.p, m.nV, 1, order);
                permute_range(order.p, 0, m.nV, {&m.isB2}, { {m.tris.p, 4L * m.nTris}, {m.elems.p, 8L * m.nE} }, m.nV);
                m.nSurf = nS;
            }
            const int nI = m.nV - m.nSurf;
            if (nI > 0) {
                DBuf<uint32_t> ks(56L * m.nE, s), vs(56L * m.nE, s);
                DBuf<int> cnt(1, s);
                cnt.zero();
                k_hex_pairs<<<G(m.nE), 256, 0, s>>>(m.elems.p, m.nE, m.nSurf, nI, ks.p, vs.p, cnt.p);
                VSDMO_CHECK_LAUNCH();
                int np = read_scalar(cnt.p, s);
                m.nColInner = color_range(m.nSurf, nI, ks, vs, np, m.col_inner, m.d_col_inner, {&m.isB2},
                                          { {m.tris.p, 4L * m.nTris}, {m.elems.p, 8L * m.nE} });
            } else {
                m.nColInner = 0;
                m.col_inner.assign(1, m.nSurf);
                m.d_col_inner.alloc(1, s);
                VSDMO_CUDA(cudaMemcpyAsync(m.d_col_inner.p, m.col_inner.data(), sizeof(int), cudaMemcpyHostToDevice, s));
            }
            if (m.nSurf > 0) surface_init();
            hex_halfhexes();
        }
        m.new_of_old.alloc(m.nV, s);
        k_final_perm<<<G(m.nV), 256, 0, s>>>(orig_of_cur.p, m.nV, m.new_of_old.p);
        VSDMO_CHECK_LAUNCH();
        m.sync();
    }
};

}  // namespace

void build_mesh(Mesh& m, const float* d_xyz, const int* d_elems) {
    Builder b(m);
    b.run(d_xyz, d_elems);
}

void update_normals(const Mesh& m, cudaStream_t s) {
    if (m.nTris <= 0 || m.nSurf <= 0) return;
    k_face_normals<<<G(m.nTris), 256, 0, s>>>(m.tris.p, m.fk, m.nTris, m.pos.p, m.fn.p, nullptr);
    VSDMO_CHECK_LAUNCH();
    k_vertex_normals<<<G(m.nSurf), 256, 0, s>>>(m.nSurf, m.he_rowptr.p, m.he.p, m.fn.p, m.vn.p);
    VSDMO_CHECK_LAUNCH();
}

}  // namespace vsdmo
