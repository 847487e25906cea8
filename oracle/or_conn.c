/*
 * or_conn.c -- CPU restatement of the reference's connectivity build and vertex colouring
 * (TEST INFRASTRUCTURE ONLY; see vsdmo_oracle.h).
 *
 * Follows, in order of execution:
 *   MeshTetGPU::init                      mesh/MeshTetGPU.cu:35-42
 *     initBoundary2D                      mesh/MeshTetGPU.cu:178-200
 *       k_constructTrisFromTetrahedra     mesh/MeshGPUCommon.cu:1398-1410 (+ :1371-1381)
 *       removeNonBoundaryTriangles        mesh/MeshTetGPU.cu:93-109, k_markDuplicateTris :56-74
 *       k_setBoundary2DVertices           mesh/MeshGPUCommon.cu:497-504
 *     colorInnerVerticesAndSort           mesh/MeshTetGPU.cu:298-392
 *       sortVerticesByBoundary2D          mesh/MeshTetGPU.cu:241-262 (stable radix, true first)
 *       constructSimpleFulledgesInnerNew  mesh/MeshTetGPU.cu:460-506, emitter MeshGPUCommon.cu:858-872
 *       colouring                         see or_color_jpl below
 *       sortInnerVerticesRangeByColor     mesh/MeshTetGPU.cu:264-295, reindex SortUtil.cu:121-144
 *   MeshTriGPU::init                      mesh/MeshTriGPU.cu:37-50
 *     calcFaceNormals                     mesh/MeshGPUCommon.cu:363-386
 *     initBoundary1DAndFeaturesNew        mesh/MeshTriGPU.cu:463-510, k_initBoundary1DRowPtr
 *                                         MeshGPUCommon.cu:1227-1239, k_initFeaturesRowPtr :466-495
 *     colorVerticesAndSort                mesh/MeshTriGPU.cu:690-784 (tet overrides of the adjacency
 *                                         emitters MeshTetGPU.cu:509-604, MeshGPUCommon.cu:874-904;
 *                                         tri emitters MeshGPUCommon.cu:1042-1064)
 *     constructTriHalfedgesNew            mesh/MeshTriGPU.cu:128-214 with k_constructHalfedges1New
 *                                         :577-595, k_setOppositeHalfedgeHelper :107-121,
 *                                         k_addBoundaryHalfedges :565-575, k_sortCCWDummyOpposite
 *                                         :211-285, k_setNextHalfedgeHelper :123-135
 *     calcVertexNormals                   mesh/MeshGPUCommon.cu:413-434
 *   constructHalffacesNew                 mesh/MeshTetGPU.cu:113-142, k_constructHalffacesNew
 *                                         MeshGPUCommon.cu:1313-1332
 *
 * Row pointers are plain CSR offsets (the intended result of k_find_first_n, SortUtil.cu:3-35).
 * Colouring: the reference's live path calls the closed cusparseScsrcolor
 * (mesh/VertexColoring.cu:128-153), whose result cannot be restated. The build uses the
 * reference's own Jones-Plassmann-Luby round rule (k_color_jpl_kernel, VertexColoring.cu:76-105:
 * an uncoloured vertex is coloured in round c iff its priority beats every neighbour that is
 * uncoloured or coloured in round c) with priorities from a seeded 32-bit bijective hash instead
 * of the index-based priorities of VertexColoring.cu:54-72/107-125 (those make every round colour
 * a single vertex on structured meshes, i.e. one colour per vertex); by default the vertex takes
 * the smallest colour its coloured neighbours do not have, with OR_COLOR_ROUNDS in the seed (and
 * with OR_COLOR_REFERENCE) the round itself, as the reference does.
 */
#include "vsdmo_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <math.h>
#include <limits.h>

struct or_mesh {
    int type, nV, nE, k;
    int nSurf, nFeature, nTris, nHE;
    int nColFree, nColFeature, nColInner;
    int maxHE, maxTets, isFlat;
    int fk;           /* vertices per surface face: 3 (tri / tet boundary) or 4 (quad) */
    float* xyz;
    int* new_of_old;
    int* elems;
    int* tris;
    int* he_rowptr;
    int* he;          /* [nHE*4] */
    int* hf_rowptr;
    int* hf;          /* [4nT*3] */
    int* col_free;
    int* col_feature;
    int* col_inner;
    uint8_t* isB1;
    uint8_t* isFeat;
    uint8_t* isB2;
    float* fn;
    float* vn;
};

#define ERR(...) do { if (err) snprintf(err, err_len, __VA_ARGS__); goto fail; } while (0)

static void* xc(size_t n, size_t s) { void* p = calloc(n ? n : 1, s); if (!p) abort(); return p; }

uint32_t or_priority(uint32_t i, uint32_t seed) {
    uint32_t h = i + seed * 0x9E3779B9u;
    h ^= h >> 16; h *= 0x85EBCA6Bu;
    h ^= h >> 13; h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

/* Round c colours every uncoloured vertex whose priority beats all its neighbours that are
 * uncoloured or coloured in round c (rnd: the round of each vertex, -1 before). The colour is c
 * (round colours: OR_COLOR_REFERENCE and OR_COLOR_ROUNDS seeds) or, by default, the smallest
 * colour that none of the vertex's coloured neighbours has (all of them have higher priorities),
 * i.e. the greedy colouring in priority order. Returns the number of colours. */
int or_color_jpl(int n, const int32_t* rowptr, const int32_t* col, uint32_t seed, int32_t* colors) {
    uint32_t* pr = (uint32_t*)xc((size_t)n, sizeof(uint32_t));
    uint8_t* win = (uint8_t*)xc((size_t)n, 1);
    int* rnd = (int*)xc((size_t)n, sizeof(int));
    const int first_fit = seed != OR_COLOR_REFERENCE && !(seed & OR_COLOR_ROUNDS);
    for (int i = 0; i < n; ++i) {
        /* OR_COLOR_REFERENCE: the reference's priorities randoms[i] = n - i (VertexColoring.cu:112) */
        pr[i] = seed == OR_COLOR_REFERENCE ? (uint32_t)(n - i) : or_priority((uint32_t)i, seed & ~OR_COLOR_ROUNDS);
        colors[i] = -1;
        rnd[i] = -1;
    }
    int left = n, c = 0, ncol = 0;
    while (left > 0) {
        for (int i = 0; i < n; ++i) {
            win[i] = 0;
            if (rnd[i] != -1) continue;
            int f = 1;
            for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
                int j = col[e];
                int jr = rnd[j];
                if ((jr != -1 && jr != c) || i == j) continue;
                if (pr[i] <= pr[j]) { f = 0; break; }
            }
            win[i] = (uint8_t)f;
        }
        for (int i = 0; i < n; ++i) {
            if (!win[i]) continue;
            int colour = c;
            if (first_fit) {
                for (colour = 0;; ++colour) {
                    int taken = 0;
                    for (int e = rowptr[i]; e < rowptr[i + 1] && !taken; ++e) {
                        int j = col[e];
                        taken = j != i && rnd[j] != -1 && rnd[j] != c && colors[j] == colour;
                    }
                    if (!taken) break;
                }
            }
            colors[i] = colour;
            if (colour + 1 > ncol) ncol = colour + 1;
            --left;
        }
        for (int i = 0; i < n; ++i) if (win[i]) rnd[i] = c;
        ++c;
    }
    free(pr); free(win); free(rnd);
    return first_fit ? ncol : c;
}

/* stable order (new -> old) putting elements with flag == first_value first */
static void stable_partition(int n, const uint8_t* flag, int first_value, int* order) {
    int p = 0;
    for (int i = 0; i < n; ++i) if ((flag[i] != 0) == (first_value != 0)) order[p++] = i;
    for (int i = 0; i < n; ++i) if ((flag[i] != 0) != (first_value != 0)) order[p++] = i;
}

/* stable counting sort of keys in [0,K): order (new -> old) and CSR offsets [K+1] */
static void counting_sort(int n, const int* keys, int K, int* order, int* offs) {
    int* cnt = (int*)xc((size_t)K + 1, sizeof(int));
    for (int i = 0; i < n; ++i) cnt[keys[i] + 1]++;
    for (int k = 0; k < K; ++k) cnt[k + 1] += cnt[k];
    if (offs) memcpy(offs, cnt, sizeof(int) * ((size_t)K + 1));
    for (int i = 0; i < n; ++i) order[cnt[keys[i]]++] = i;
    free(cnt);
}

static int cmp_int(const void* a, const void* b) {
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* adjacency CSR (sorted unique rows) from an edge pair list */
static void build_adjacency(int n, int npairs, const int* src, const int* dst, int** rowptr_out, int** col_out) {
    int* rowptr = (int*)xc((size_t)n + 1, sizeof(int));
    for (int e = 0; e < npairs; ++e) rowptr[src[e] + 1]++;
    for (int i = 0; i < n; ++i) rowptr[i + 1] += rowptr[i];
    int* fill = (int*)xc((size_t)n + 1, sizeof(int));
    memcpy(fill, rowptr, sizeof(int) * ((size_t)n + 1));
    int* col = (int*)xc((size_t)npairs, sizeof(int));
    for (int e = 0; e < npairs; ++e) col[fill[src[e]]++] = dst[e];
    /* sort + unique per row, compact */
    int w = 0;
    int* newrow = (int*)xc((size_t)n + 1, sizeof(int));
    for (int i = 0; i < n; ++i) {
        int b = rowptr[i], e = rowptr[i + 1];
        qsort(col + b, (size_t)(e - b), sizeof(int), cmp_int);
        newrow[i] = w;
        for (int j = b; j < e; ++j) {
            if (j > b && col[j] == col[j - 1]) continue;
            col[w++] = col[j];
        }
    }
    newrow[n] = w;
    free(rowptr); free(fill);
    *rowptr_out = newrow;
    *col_out = col;
}

/* ---- vertex permutation bookkeeping ---------------------------------------------------- */
typedef struct {
    int nV;
    float* xyz;
    int* old_of_cur;   /* current index -> original index */
} vstate;

/* apply order (new->old) restricted to range [start, start+num): permute xyz / flags and
 * return inv (old->new over the whole range [0, nTot)) so element indices can be remapped */
static void permute_range(int start, int num, const int* order_local, float* xyz, int* old_of_cur,
                          uint8_t* f1, uint8_t* f2, uint8_t* f3, int* inv, int nTot) {
    for (int i = 0; i < nTot; ++i) inv[i] = i;
    float* tx = (float*)xc((size_t)num * 3, sizeof(float));
    int* to = (int*)xc((size_t)num, sizeof(int));
    uint8_t* t1 = (uint8_t*)xc((size_t)num, 1);
    uint8_t* t2 = (uint8_t*)xc((size_t)num, 1);
    uint8_t* t3 = (uint8_t*)xc((size_t)num, 1);
    for (int i = 0; i < num; ++i) {
        int o = start + order_local[i];
        inv[o] = start + i;
        memcpy(tx + 3 * i, xyz + 3 * (size_t)o, 3 * sizeof(float));
        to[i] = old_of_cur[o];
        if (f1) t1[i] = f1[o];
        if (f2) t2[i] = f2[o];
        if (f3) t3[i] = f3[o];
    }
    memcpy(xyz + 3 * (size_t)start, tx, sizeof(float) * 3 * (size_t)num);
    memcpy(old_of_cur + start, to, sizeof(int) * (size_t)num);
    if (f1) memcpy(f1 + start, t1, (size_t)num);
    if (f2) memcpy(f2 + start, t2, (size_t)num);
    if (f3) memcpy(f3 + start, t3, (size_t)num);
    free(tx); free(to); free(t1); free(t2); free(t3);
}

static void remap(int n, int* idx, const int* inv, int nInv) {
    for (int i = 0; i < n; ++i) if (idx[i] >= 0 && idx[i] < nInv) idx[i] = inv[idx[i]];
}

/* colour one vertex range [start, start+num) with the given pair list (local indices) and
 * sort it by colour; returns number of colours and fills offsets (absolute, +start) */
static int color_and_sort_range(int start, int num, int npairs, const int* ps, const int* pd,
                                uint32_t seed, float* xyz, int* old_of_cur, uint8_t* f1, uint8_t* f2,
                                uint8_t* f3, int nTot, int* elemsA, int nA, int* elemsB, int nB,
                                int** offs_out) {
    int* rowptr; int* col;
    build_adjacency(num, npairs, ps, pd, &rowptr, &col);
    int* colors = (int*)xc((size_t)num, sizeof(int));
    int nc = or_color_jpl(num, rowptr, col, seed, colors);
    /* dense reindex of used colours (SortUtil.cu:121-144) */
    int* used = (int*)xc((size_t)nc + 1, sizeof(int));
    for (int i = 0; i < num; ++i) used[colors[i]] = 1;
    int* map = (int*)xc((size_t)nc + 1, sizeof(int));
    int cur = 0;
    for (int c = 0; c < nc; ++c) if (used[c]) map[c] = cur++;
    for (int i = 0; i < num; ++i) colors[i] = map[colors[i]];
    nc = cur;
    int* order = (int*)xc((size_t)num, sizeof(int));
    int* offs = (int*)xc((size_t)nc + 1, sizeof(int));
    counting_sort(num, colors, nc, order, offs);
    for (int c = 0; c <= nc; ++c) offs[c] += start;
    int* inv = (int*)xc((size_t)nTot, sizeof(int));
    permute_range(start, num, order, xyz, old_of_cur, f1, f2, f3, inv, nTot);
    if (elemsA) remap(nA, elemsA, inv, nTot);
    if (elemsB) remap(nB, elemsB, inv, nTot);
    free(rowptr); free(col); free(colors); free(used); free(map); free(order); free(inv);
    *offs_out = offs;
    return nc;
}

/* ---- surface halfedges ----------------------------------------------------------------- */
static int third_vertex_tri(const int* t, int src, int dst) {
    if (t[0] != src && t[0] != dst) return t[0];
    if (t[1] != src && t[1] != dst) return t[1];
    return t[2];
}

/* getThirdVertex for quads (mesh/MeshGPUCommon.cu:149-162): the corner two after dst */
static int third_vertex_quad(const int* q, int src, int dst) {
    (void)src;
    if (dst == q[1]) return q[3];
    if (dst == q[2]) return q[0];
    if (dst == q[3]) return q[1];
    return q[2];
}

static void calc_face_normals(int nTris, int fk, const int* tris, const float* xyz, float* fn, int* bad) {
    for (int t = 0; t < nTris; ++t) {
        const float* p0 = xyz + 3 * (size_t)tris[fk * t];
        const float* p1 = xyz + 3 * (size_t)tris[fk * t + 1];
        const float* p2 = xyz + 3 * (size_t)tris[fk * t + (fk == 4 ? 3 : 2)];
        float e0[3] = { p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2] };
        float e1[3] = { p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2] };
        float l0 = sqrtf(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
        float l1 = sqrtf(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
        if (bad && (l0 < 1e-6f || l1 < 1e-6f)) *bad = 1;
        float n[3] = { e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0] };
        float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        fn[3 * t] = n[0] / len; fn[3 * t + 1] = n[1] / len; fn[3 * t + 2] = n[2] / len;
    }
}

/* first-pass halfedges (no dummies): rows by src in triangle order; he4[i] = {target,opp,face,next} */
static void first_halfedges(int nS, int nTris, int fk, const int* tris, int** rowptr_out, int** he_out) {
    int nHE = fk * nTris;
    int* keys = (int*)xc((size_t)nHE, sizeof(int));
    for (int t = 0; t < nTris; ++t) for (int j = 0; j < fk; ++j) keys[fk * t + j] = tris[fk * t + j];
    int* order = (int*)xc((size_t)nHE, sizeof(int));
    int* rowptr = (int*)xc((size_t)nS + 1, sizeof(int));
    counting_sort(nHE, keys, nS, order, rowptr);
    int* he = (int*)xc((size_t)nHE * 4, sizeof(int));
    for (int i = 0; i < nHE; ++i) {
        int e = order[i], t = e / fk, j = e % fk;
        he[4 * i] = tris[fk * t + (j + 1) % fk];
        he[4 * i + 1] = -1; he[4 * i + 2] = t; he[4 * i + 3] = 0;
    }
    /* opposite: last entry of target's row pointing back to src */
    for (int v = 0; v < nS; ++v)
        for (int i = rowptr[v]; i < rowptr[v + 1]; ++i) {
            int dst = he[4 * i], opp = -1;
            for (int q = rowptr[dst]; q < rowptr[dst + 1]; ++q) if (he[4 * q] == v) opp = q;
            he[4 * i + 1] = opp;
        }
    free(keys); free(order);
    *rowptr_out = rowptr; *he_out = he;
}

static int final_halfedges(or_mesh* m, int nS, char* err, int err_len) {
    int* r1; int* h1;
    first_halfedges(nS, m->nTris, m->fk, m->tris, &r1, &h1);
    int nHE1 = m->fk * m->nTris;
    /* dummies: for every halfedge without opposite, a reversed one with face -1, keyed by its
     * target, appended after all real ones in sorted order (stable sort keeps that order) */
    int nD = 0;
    for (int i = 0; i < nHE1; ++i) if (h1[4 * i + 1] == -1) nD++;
    int nHE = nHE1 + nD;
    int* keys = (int*)xc((size_t)nHE, sizeof(int));
    int* tmp = (int*)xc((size_t)nHE * 4, sizeof(int));
    int w = 0;
    for (int v = 0; v < nS; ++v) for (int i = r1[v]; i < r1[v + 1]; ++i) {
        keys[w] = v; memcpy(tmp + 4 * w, h1 + 4 * i, 4 * sizeof(int)); w++;
    }
    for (int v = 0; v < nS; ++v) for (int i = r1[v]; i < r1[v + 1]; ++i) if (h1[4 * i + 1] == -1) {
        keys[w] = h1[4 * i]; tmp[4 * w] = v; tmp[4 * w + 1] = -1; tmp[4 * w + 2] = -1; tmp[4 * w + 3] = 0; w++;
    }
    int* order = (int*)xc((size_t)nHE, sizeof(int));
    int* rowptr = (int*)xc((size_t)nS + 1, sizeof(int));
    counting_sort(nHE, keys, nS, order, rowptr);
    int* in = (int*)xc((size_t)nHE * 4, sizeof(int));
    for (int i = 0; i < nHE; ++i) memcpy(in + 4 * i, tmp + 4 * order[i], 4 * sizeof(int));
    for (int v = 0; v < nS; ++v) for (int i = rowptr[v]; i < rowptr[v + 1]; ++i) {
        int dst = in[4 * i], opp = -1;
        for (int q = rowptr[dst]; q < rowptr[dst + 1]; ++q) if (in[4 * q] == v) opp = q;
        in[4 * i + 1] = opp;
    }
    int* out = (int*)xc((size_t)nHE * 4, sizeof(int));
    for (int src = 0; src < nS; ++src) {
        int start = rowptr[src], n = rowptr[src + 1] - start, outPos = 0;
        if (n == 0) ERR("vertex %d has no halfedges", src);
        int h[4]; memcpy(h, in + 4 * start, sizeof h);
        if (m->isB1[src]) {
            int j = 0;
            while (1) {
                if (h[1] < 0) ERR("boundary halfedge without opposite at vertex %d", src);
                if (in[4 * h[1] + 2] == -1) break;
                if (++j == n) ERR("non-manifold boundary fan at vertex %d", src);
                memcpy(h, in + 4 * (start + j), sizeof h);
            }
        } else if (m->isFeat[src]) {
            h[0] = INT_MAX;
            for (int j = 0; j < n; ++j) {
                const int* t = in + 4 * (start + j);
                if (m->isFeat[t[0]] && t[0] < h[0]) memcpy(h, t, sizeof h);
            }
            if (h[0] == INT_MAX) ERR("feature vertex %d without feature neighbour", src);
        } else {
            for (int i = 1; i < n; ++i) if (in[4 * (start + i)] < h[0]) memcpy(h, in + 4 * (start + i), sizeof h);
        }
        memcpy(out + 4 * (start + outPos), h, sizeof h); ++outPos;
        int found;
        do {
            int currDst = h[0], currTri = h[2];
            if (currTri == -1) ERR("fan walk reached a boundary at vertex %d", src);
            int nextVert = m->fk == 4 ? third_vertex_quad(m->tris + 4 * (size_t)currTri, src, currDst)
                                      : third_vertex_tri(m->tris + 3 * (size_t)currTri, src, currDst);
            found = 0;
            for (int j = 0; j < n; ++j) if (in[4 * (start + j)] == nextVert) {
                if (outPos >= n) ERR("non-manifold fan at vertex %d", src);
                found = 1; memcpy(h, in + 4 * (start + j), sizeof h);
                memcpy(out + 4 * (start + outPos), h, sizeof h); ++outPos;
            }
        } while (found && outPos < n);
        if (outPos != n) ERR("open fan at vertex %d (%d of %d halfedges)", src, outPos, n);
    }
    for (int v = 0; v < nS; ++v) for (int i = rowptr[v]; i < rowptr[v + 1]; ++i) {
        int dst = out[4 * i], opp = -1, nxt = out[4 * i + 3];
        for (int q = rowptr[dst]; q < rowptr[dst + 1]; ++q) if (out[4 * q] == v) opp = q;
        out[4 * i + 1] = opp;
        for (int q = rowptr[dst]; q < rowptr[dst + 1]; ++q) if (out[4 * q + 2] == out[4 * i + 2]) nxt = q;
        out[4 * i + 3] = nxt;
    }
    int mx = 0;
    for (int v = 0; v < nS; ++v) if (rowptr[v + 1] - rowptr[v] > mx) mx = rowptr[v + 1] - rowptr[v];
    m->maxHE = mx;
    m->nHE = nHE;
    m->he_rowptr = rowptr;
    m->he = out;
    free(r1); free(h1); free(keys); free(tmp); free(order); free(in);
    return 0;
fail:
    free(r1); free(h1); free(keys); free(tmp); free(order); free(in); free(out); free(rowptr);
    return -1;
}

static void calc_vertex_normals(or_mesh* m, int nS) {
    for (int v = 0; v < nS; ++v) {
        float n[3] = { 0.f, 0.f, 0.f };
        for (int i = m->he_rowptr[v]; i < m->he_rowptr[v + 1]; ++i) {
            int f = m->he[4 * i + 2];
            if (f != -1) { n[0] += m->fn[3 * f]; n[1] += m->fn[3 * f + 1]; n[2] += m->fn[3 * f + 2]; }
        }
        float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        m->vn[3 * v] = n[0] / len; m->vn[3 * v + 1] = n[1] / len; m->vn[3 * v + 2] = n[2] / len;
    }
}

/* surface initialisation shared by tri meshes and the boundary of tet meshes */
static int surface_init(or_mesh* m, int* old_of_cur, uint32_t seed, char* err, int err_len) {
    int nS = m->nSurf;
    int bad = 0;
    m->fn = (float*)xc((size_t)m->nTris * 3, sizeof(float));
    calc_face_normals(m->nTris, m->fk, m->tris, m->xyz, m->fn, &bad);
    if (bad) { if (err) snprintf(err, err_len, "degenerate triangle (edge shorter than 1e-6)"); return -1; }
    int* r1; int* h1;
    first_halfedges(nS, m->nTris, m->fk, m->tris, &r1, &h1);
    m->isB1 = (uint8_t*)xc((size_t)nS, 1);
    m->isFeat = (uint8_t*)xc((size_t)nS, 1);
    for (int v = 0; v < nS; ++v)
        for (int i = r1[v]; i < r1[v + 1]; ++i) if (h1[4 * i + 1] == -1) { m->isB1[v] = 1; break; }
    if (m->isFlat) {
        memcpy(m->isFeat, m->isB1, (size_t)nS);
    } else {
        for (int v = 0; v < nS; ++v)
            for (int i = r1[v]; i < r1[v + 1]; ++i) {
                int dst = h1[4 * i], opp = h1[4 * i + 1];
                if (opp == -1) { m->isFeat[v] = 1; m->isFeat[dst] = 1; continue; }
                const float* f1 = m->fn + 3 * (size_t)h1[4 * i + 2];
                const float* f2 = m->fn + 3 * (size_t)h1[4 * opp + 2];
                float dot = f1[0] * f2[0] + f1[1] * f2[1] + f1[2] * f2[2];
                float len = sqrtf((f1[0] * f1[0] + f1[1] * f1[1] + f1[2] * f1[2]) * (f2[0] * f2[0] + f2[1] * f2[1] + f2[2] * f2[2]));
                /* a float angle, as in the reference (MeshGPUCommon.cu:485-488) */
                float angle = (float)(180.0 / M_PI * (double)acosf(dot / len));
                if (angle > 20.f) { m->isFeat[v] = 1; m->isFeat[dst] = 1; }
            }
    }
    free(r1); free(h1);
    /* free vertices first, feature vertices last (stable) */
    int* order = (int*)xc((size_t)nS, sizeof(int));
    stable_partition(nS, m->isFeat, 0, order);
    int nTot = m->nV;
    int* inv = (int*)xc((size_t)nTot, sizeof(int));
    permute_range(0, nS, order, m->xyz, old_of_cur, m->isB1, m->isFeat, NULL, inv, nTot);
    remap(m->nTris * m->fk, m->tris, inv, nS);
    if (m->type == OR_TET || m->type == OR_HEX) remap(m->nE * m->k, m->elems, inv, nS);
    free(order); free(inv);
    int nFree = 0;
    for (int v = 0; v < nS; ++v) if (!m->isFeat[v]) nFree++;
    m->nFeature = nS - nFree;
    /* adjacency pairs for the two partitions */
    for (int part = 0; part < 2; ++part) {
        int lo = part == 0 ? 0 : nFree, hi = part == 0 ? nFree : nS;
        int num = hi - lo;
        if (num <= 0) {
            int* offs = (int*)xc(1, sizeof(int)); offs[0] = lo;
            if (part == 0) { m->col_free = offs; m->nColFree = 0; }
            else { m->col_feature = offs; m->nColFeature = 0; }
            continue;
        }
        int cap = m->type == OR_TET ? 12 * m->nE : m->type == OR_HEX ? 56 * m->nE : (m->fk == 4 ? 12 : 6) * m->nTris;
        int* ps = (int*)xc((size_t)cap, sizeof(int));
        int* pd = (int*)xc((size_t)cap, sizeof(int));
        int np = 0;
        if (m->type == OR_HEX) {
            /* every vertex pair of a hexahedron (mesh/MeshGPUCommon.cu:982-1037) */
            for (int t = 0; t < m->nE; ++t)
                for (int i = 0; i < 7; ++i)
                    for (int j = i + 1; j < 8; ++j) {
                        int a = m->elems[8 * t + i] - lo, b = m->elems[8 * t + j] - lo;
                        if (a >= 0 && a < num && b >= 0 && b < num) { ps[np] = a; pd[np++] = b; ps[np] = b; pd[np++] = a; }
                    }
        } else if (m->type == OR_TET) {
            static const int E[6][2] = { {0,1},{0,2},{0,3},{1,2},{1,3},{2,3} };
            for (int t = 0; t < m->nE; ++t) for (int e = 0; e < 6; ++e) {
                int a = m->elems[4 * t + E[e][0]] - lo, b = m->elems[4 * t + E[e][1]] - lo;
                if (a >= 0 && a < num && b >= 0 && b < num) { ps[np] = a; pd[np++] = b; ps[np] = b; pd[np++] = a; }
            }
        } else if (m->fk == 4) {
            /* quad edges and both diagonals (mesh/MeshGPUCommon.cu:1067-1097) */
            static const int E[6][2] = { {0,1},{1,2},{2,3},{3,0},{0,2},{1,3} };
            for (int t = 0; t < m->nTris; ++t) for (int e = 0; e < 6; ++e) {
                int a = m->tris[4 * t + E[e][0]] - lo, b = m->tris[4 * t + E[e][1]] - lo;
                if (a >= 0 && a < num && b >= 0 && b < num) { ps[np] = a; pd[np++] = b; ps[np] = b; pd[np++] = a; }
            }
        } else {
            static const int E[3][2] = { {0,1},{0,2},{1,2} };
            for (int t = 0; t < m->nTris; ++t) for (int e = 0; e < 3; ++e) {
                int a = m->tris[3 * t + E[e][0]] - lo, b = m->tris[3 * t + E[e][1]] - lo;
                if (a >= 0 && a < num && b >= 0 && b < num) { ps[np] = a; pd[np++] = b; ps[np] = b; pd[np++] = a; }
            }
        }
        int* offs;
        int nc = color_and_sort_range(lo, num, np, ps, pd, seed, m->xyz, old_of_cur, m->isB1, m->isFeat, NULL,
                                      nTot, m->tris, m->nTris * m->fk,
                                      (m->type == OR_TET || m->type == OR_HEX) ? m->elems : NULL,
                                      (m->type == OR_TET || m->type == OR_HEX) ? m->nE * m->k : 0, &offs);
        if (part == 0) { m->col_free = offs; m->nColFree = nc; }
        else { m->col_feature = offs; m->nColFeature = nc; }
        free(ps); free(pd);
    }
    if (final_halfedges(m, nS, err, err_len)) return -1;
    m->vn = (float*)xc((size_t)nS * 3, sizeof(float));
    calc_vertex_normals(m, nS);
    return 0;
}

/* ---- tetrahedral boundary --------------------------------------------------------------- */
typedef struct { int v[3]; } tri3;

static tri3 smallest_first(int a, int b, int c) {
    tri3 t;
    if (a < b && a < c) { t.v[0] = a; t.v[1] = b; t.v[2] = c; }
    else if (b < a && b < c) { t.v[0] = b; t.v[1] = c; t.v[2] = a; }
    else { t.v[0] = c; t.v[1] = a; t.v[2] = b; }
    return t;
}

typedef struct { int v[4]; } quad4;

/* getQuadSmallestFirst / k_reorderVertices for quads (mesh/MeshGPUCommon.cu:37-54) */
static quad4 quad_smallest_first(int a, int b, int c, int d) {
    quad4 q;
    if (b < a && b < c && b < d) { q.v[0] = b; q.v[1] = c; q.v[2] = d; q.v[3] = a; }
    else if (c < a && c < b && c < d) { q.v[0] = c; q.v[1] = d; q.v[2] = a; q.v[3] = b; }
    else if (d < a && d < b && d < c) { q.v[0] = d; q.v[1] = a; q.v[2] = b; q.v[3] = c; }
    else { q.v[0] = a; q.v[1] = b; q.v[2] = c; q.v[3] = d; }
    return q;
}

static int cmp_quad(const void* A, const void* B) {
    const quad4* a = (const quad4*)A; const quad4* b = (const quad4*)B;
    for (int i = 0; i < 4; ++i) { if (a->v[i] < b->v[i]) return -1; if (a->v[i] > b->v[i]) return 1; }
    return 0;
}

/* halfhex of corner j: the other seven corners (k_constructHalfhexesNew,
 * mesh/MeshGPUCommon.cu:1334-1368) */
static const int HALFHEX[8][7] = {
    { 1, 2, 3, 4, 5, 6, 7 }, { 5, 6, 2, 0, 4, 7, 3 }, { 6, 7, 3, 1, 5, 4, 0 }, { 7, 4, 0, 2, 6, 5, 1 },
    { 0, 3, 7, 5, 1, 2, 6 }, { 4, 7, 6, 1, 0, 3, 2 }, { 5, 4, 7, 2, 1, 0, 3 }, { 6, 5, 4, 3, 2, 1, 0 } };

/* MeshHexGPU::init (mesh/MeshHexGPU.cu:35-43): boundary quads, boundary-first order, interior
 * colouring, the quad surface, halfhexes */
static int build_hex(or_mesh* m, int* old_of_cur, uint32_t seed, char* err, int err_len) {
    const int nV = m->nV, nE = m->nE;
    m->fk = 4;
    int nF = 6 * nE;
    quad4* f = (quad4*)xc((size_t)nF, sizeof(quad4));
    for (int t = 0; t < nE; ++t) {
        const int* v = m->elems + 8 * t;
        f[6 * t + 0] = quad_smallest_first(v[0], v[1], v[2], v[3]);
        f[6 * t + 1] = quad_smallest_first(v[1], v[5], v[6], v[2]);
        f[6 * t + 2] = quad_smallest_first(v[3], v[2], v[6], v[7]);
        f[6 * t + 3] = quad_smallest_first(v[4], v[0], v[3], v[7]);
        f[6 * t + 4] = quad_smallest_first(v[1], v[0], v[4], v[5]);
        f[6 * t + 5] = quad_smallest_first(v[5], v[4], v[7], v[6]);
    }
    qsort(f, (size_t)nF, sizeof(quad4), cmp_quad);
    /* k_markDuplicateQuads in index order */
    for (int idx = 0; idx < nF; ++idx) {
        quad4* q = &f[idx];
        if (q->v[1] < q->v[3]) {
            for (int i = idx + 1; i < nF; ++i) {
                quad4* it = &f[i];
                if (it->v[0] > q->v[0]) break;
                if (q->v[0] == it->v[0] && q->v[1] == it->v[3] && q->v[2] == it->v[2] && q->v[3] == it->v[1]) {
                    q->v[0] = -1; it->v[0] = -1; break;
                }
            }
        }
    }
    int nB = 0;
    for (int i = 0; i < nF; ++i) if (f[i].v[0] != -1) nB++;
    m->nTris = nB;
    m->tris = (int*)xc((size_t)nB * 4, sizeof(int));
    for (int i = 0, w = 0; i < nF; ++i) if (f[i].v[0] != -1) { memcpy(m->tris + 4 * w, f[i].v, 4 * sizeof(int)); w++; }
    free(f);
    m->isB2 = (uint8_t*)xc((size_t)nV, 1);
    for (int i = 0; i < 4 * nB; ++i) m->isB2[m->tris[i]] = 1;
    int* order = (int*)xc((size_t)nV, sizeof(int));
    stable_partition(nV, m->isB2, 1, order);
    int* inv = (int*)xc((size_t)nV, sizeof(int));
    permute_range(0, nV, order, m->xyz, old_of_cur, m->isB2, NULL, NULL, inv, nV);
    remap(4 * nB, m->tris, inv, nV);
    remap(8 * nE, m->elems, inv, nV);
    free(order); free(inv);
    int nS = 0;
    for (int i = 0; i < nV; ++i) if (m->isB2[i]) nS++;
    m->nSurf = nS;
    const int nI = nV - nS;
    if (nI > 0) {
        int* ps = (int*)xc((size_t)56 * nE, sizeof(int));
        int* pd = (int*)xc((size_t)56 * nE, sizeof(int));
        int np = 0;
        for (int t = 0; t < nE; ++t)
            for (int i = 0; i < 7; ++i)
                for (int j = i + 1; j < 8; ++j) {
                    int a = m->elems[8 * t + i], b = m->elems[8 * t + j];
                    if (!m->isB2[a] && !m->isB2[b]) { ps[np] = a - nS; pd[np++] = b - nS; ps[np] = b - nS; pd[np++] = a - nS; }
                }
        m->nColInner = color_and_sort_range(nS, nI, np, ps, pd, seed, m->xyz, old_of_cur, m->isB2, NULL, NULL,
                                            nV, m->tris, 4 * nB, m->elems, 8 * nE, &m->col_inner);
        free(ps); free(pd);
    } else {
        m->col_inner = (int*)xc(1, sizeof(int)); m->col_inner[0] = nS; m->nColInner = 0;
    }
    if (nS > 0 && surface_init(m, old_of_cur, seed, err, err_len)) return -1;
    /* halfhexes: stable by vertex => rows in hexahedron order */
    const int nH = 8 * nE;
    int* keys = (int*)xc((size_t)nH, sizeof(int));
    for (int i = 0; i < nH; ++i) keys[i] = m->elems[i];
    int* ord = (int*)xc((size_t)nH, sizeof(int));
    m->hf_rowptr = (int*)xc((size_t)nV + 1, sizeof(int));
    counting_sort(nH, keys, nV, ord, m->hf_rowptr);
    m->hf = (int*)xc((size_t)nH * 7, sizeof(int));
    for (int i = 0; i < nH; ++i) {
        const int t = ord[i] / 8, j = ord[i] % 8;
        const int* v = m->elems + 8 * t;
        for (int a = 0; a < 7; ++a) m->hf[7 * i + a] = v[HALFHEX[j][a]];
    }
    int mx = 0;
    for (int v = 0; v < nV; ++v) if (m->hf_rowptr[v + 1] - m->hf_rowptr[v] > mx) mx = m->hf_rowptr[v + 1] - m->hf_rowptr[v];
    m->maxTets = mx;
    free(keys); free(ord);
    return 0;
}

static int cmp_tri(const void* A, const void* B) {
    const tri3* a = (const tri3*)A; const tri3* b = (const tri3*)B;
    for (int i = 0; i < 3; ++i) { if (a->v[i] < b->v[i]) return -1; if (a->v[i] > b->v[i]) return 1; }
    return 0;
}

or_mesh* or_mesh_build(int elem_type, int nV, const float* xyz, int nE, const int32_t* elems,
                       uint32_t seed, char* err, int err_len) {
    if (err && err_len > 0) err[0] = 0;
    if (elem_type != OR_TRI && elem_type != OR_TET && elem_type != OR_QUAD && elem_type != OR_HEX) { if (err) snprintf(err, err_len, "element type not supported by the oracle"); return NULL; }
    if (nV <= 0 || nE <= 0 || !xyz || !elems) { if (err) snprintf(err, err_len, "empty mesh"); return NULL; }
    int k = elem_type == OR_TRI ? 3 : elem_type == OR_HEX ? 8 : 4;
    for (long i = 0; i < (long)nE * k; ++i) if (elems[i] < 0 || elems[i] >= nV) { if (err) snprintf(err, err_len, "element index out of range"); return NULL; }
    or_mesh* m = (or_mesh*)xc(1, sizeof(or_mesh));
    m->type = elem_type; m->nV = nV; m->nE = nE; m->k = k;
    m->xyz = (float*)xc((size_t)nV * 3, sizeof(float));
    memcpy(m->xyz, xyz, sizeof(float) * 3 * (size_t)nV);
    m->elems = (int*)xc((size_t)nE * k, sizeof(int));
    memcpy(m->elems, elems, sizeof(int) * (size_t)nE * k);
    int* old_of_cur = (int*)xc((size_t)nV, sizeof(int));
    for (int i = 0; i < nV; ++i) old_of_cur[i] = i;
    if (elem_type == OR_TRI || elem_type == OR_QUAD) {
        m->fk = k;
        m->isFlat = 1;
        for (int i = 0; i < nV; ++i) if (xyz[3 * i + 2] != 0.f) { m->isFlat = 0; break; }
        m->nSurf = nV; m->nTris = nE;
        m->tris = (int*)xc((size_t)nE * k, sizeof(int));
        memcpy(m->tris, m->elems, sizeof(int) * k * (size_t)nE);
        m->col_inner = (int*)xc(1, sizeof(int)); m->col_inner[0] = nV;
        if (surface_init(m, old_of_cur, seed, err, err_len)) goto fail;
        memcpy(m->elems, m->tris, sizeof(int) * k * (size_t)nE);
    } else if (elem_type == OR_HEX) {
        if (build_hex(m, old_of_cur, seed, err, err_len)) goto fail;
    } else {
        m->fk = 3;
        int nF = 4 * nE;
        tri3* f = (tri3*)xc((size_t)nF, sizeof(tri3));
        for (int t = 0; t < nE; ++t) {
            const int* v = m->elems + 4 * t;
            f[4 * t + 0] = smallest_first(v[2], v[1], v[0]);
            f[4 * t + 1] = smallest_first(v[0], v[1], v[3]);
            f[4 * t + 2] = smallest_first(v[1], v[2], v[3]);
            f[4 * t + 3] = smallest_first(v[0], v[3], v[2]);
        }
        qsort(f, (size_t)nF, sizeof(tri3), cmp_tri);
        /* k_markDuplicateTris, executed in index order */
        for (int idx = 0; idx < nF; ++idx) {
            tri3* t = &f[idx];
            if (t->v[1] < t->v[2]) {
                for (int i = idx + 1; i < nF; ++i) {
                    tri3* it = &f[i];
                    if (it->v[0] > t->v[0]) break;
                    if (t->v[0] == it->v[0] && t->v[1] == it->v[2] && t->v[2] == it->v[1]) { t->v[0] = -1; it->v[0] = -1; break; }
                }
            }
        }
        int nB = 0;
        for (int i = 0; i < nF; ++i) if (f[i].v[0] != -1) nB++;
        m->nTris = nB;
        m->tris = (int*)xc((size_t)nB * 3, sizeof(int));
        for (int i = 0, w = 0; i < nF; ++i) if (f[i].v[0] != -1) { memcpy(m->tris + 3 * w, f[i].v, 3 * sizeof(int)); w++; }
        free(f);
        m->isB2 = (uint8_t*)xc((size_t)nV, 1);
        for (int i = 0; i < 3 * nB; ++i) m->isB2[m->tris[i]] = 1;
        /* boundary vertices first (stable) */
        int* order = (int*)xc((size_t)nV, sizeof(int));
        stable_partition(nV, m->isB2, 1, order);
        int* inv = (int*)xc((size_t)nV, sizeof(int));
        permute_range(0, nV, order, m->xyz, old_of_cur, m->isB2, NULL, NULL, inv, nV);
        remap(3 * nB, m->tris, inv, nV);
        remap(4 * nE, m->elems, inv, nV);
        free(order); free(inv);
        int nS = 0;
        for (int i = 0; i < nV; ++i) if (m->isB2[i]) nS++;
        m->nSurf = nS;
        int nI = nV - nS;
        if (nI > 0) {
            int* ps = (int*)xc((size_t)12 * nE, sizeof(int));
            int* pd = (int*)xc((size_t)12 * nE, sizeof(int));
            int np = 0;
            static const int E[6][2] = { {0,1},{0,2},{0,3},{1,2},{1,3},{2,3} };
            for (int t = 0; t < nE; ++t) for (int e = 0; e < 6; ++e) {
                int a = m->elems[4 * t + E[e][0]], b = m->elems[4 * t + E[e][1]];
                if (!m->isB2[a] && !m->isB2[b]) { ps[np] = a - nS; pd[np++] = b - nS; ps[np] = b - nS; pd[np++] = a - nS; }
            }
            m->nColInner = color_and_sort_range(nS, nI, np, ps, pd, seed, m->xyz, old_of_cur, m->isB2, NULL, NULL,
                                                nV, m->tris, 3 * nB, m->elems, 4 * nE, &m->col_inner);
            free(ps); free(pd);
        } else {
            m->col_inner = (int*)xc(1, sizeof(int)); m->col_inner[0] = nS; m->nColInner = 0;
        }
        if (nS > 0 && surface_init(m, old_of_cur, seed, err, err_len)) goto fail;
        /* halffaces: stable by vertex => rows in tetrahedron order */
        int nH = 4 * nE;
        int* keys = (int*)xc((size_t)nH, sizeof(int));
        for (int i = 0; i < nH; ++i) keys[i] = m->elems[i];
        int* ord = (int*)xc((size_t)nH, sizeof(int));
        m->hf_rowptr = (int*)xc((size_t)nV + 1, sizeof(int));
        counting_sort(nH, keys, nV, ord, m->hf_rowptr);
        m->hf = (int*)xc((size_t)nH * 3, sizeof(int));
        for (int i = 0; i < nH; ++i) {
            int t = ord[i] / 4, j = ord[i] % 4;
            const int* v = m->elems + 4 * t;
            int* o = m->hf + 3 * i;
            if (j == 0) { o[0] = v[1]; o[1] = v[2]; o[2] = v[3]; }
            else if (j == 1) { o[0] = v[0]; o[1] = v[3]; o[2] = v[2]; }
            else if (j == 2) { o[0] = v[0]; o[1] = v[1]; o[2] = v[3]; }
            else { o[0] = v[0]; o[1] = v[2]; o[2] = v[1]; }
        }
        int mx = 0;
        for (int v = 0; v < nV; ++v) if (m->hf_rowptr[v + 1] - m->hf_rowptr[v] > mx) mx = m->hf_rowptr[v + 1] - m->hf_rowptr[v];
        m->maxTets = mx;
        free(keys); free(ord);
    }
    m->new_of_old = (int*)xc((size_t)nV, sizeof(int));
    for (int i = 0; i < nV; ++i) m->new_of_old[old_of_cur[i]] = i;
    free(old_of_cur);
    return m;
fail:
    free(old_of_cur);
    or_mesh_free(m);
    return NULL;
}

void or_mesh_free(or_mesh* m) {
    if (!m) return;
    free(m->xyz); free(m->new_of_old); free(m->elems); free(m->tris); free(m->he_rowptr); free(m->he);
    free(m->hf_rowptr); free(m->hf); free(m->col_free); free(m->col_feature); free(m->col_inner);
    free(m->isB1); free(m->isFeat); free(m->isB2); free(m->fn); free(m->vn);
    free(m);
}

int or_mesh_info(const or_mesh* m, int which) {
    switch (which) {
    case OR_I_NV: return m->nV;
    case OR_I_NE: return m->nE;
    case OR_I_NSURF: return m->nSurf;
    case OR_I_NFEATURE: return m->nFeature;
    case OR_I_NTRIS: return m->nTris;
    case OR_I_NHE: return m->nHE;
    case OR_I_NCOL_FREE: return m->nColFree;
    case OR_I_NCOL_FEATURE: return m->nColFeature;
    case OR_I_NCOL_INNER: return m->nColInner;
    case OR_I_MAX_HE: return m->maxHE;
    case OR_I_MAX_TETS: return m->maxTets;
    case OR_I_IS_FLAT: return m->isFlat;
    default: return -1;
    }
}

long or_mesh_array_len(const or_mesh* m, int id) {
    switch (id) {
    case OR_A_XYZ: return 3L * m->nV;
    case OR_A_NEW_OF_OLD: return m->nV;
    case OR_A_ELEMS: return (long)m->nE * m->k;
    case OR_A_SURF_TRIS: return (long)m->fk * m->nTris;
    case OR_A_HE_ROWPTR: return m->he_rowptr ? m->nSurf + 1L : 0;
    case OR_A_HALFEDGES: return 4L * m->nHE;
    case OR_A_HF_ROWPTR: return m->hf_rowptr ? m->nV + 1L : 0;
    case OR_A_HALFFACES: return m->hf ? (m->type == OR_HEX ? 56L : 12L) * m->nE : 0;
    case OR_A_COL_FREE: return m->col_free ? m->nColFree + 1L : 0;
    case OR_A_COL_FEATURE: return m->col_feature ? m->nColFeature + 1L : 0;
    case OR_A_COL_INNER: return m->col_inner ? m->nColInner + 1L : 0;
    case OR_A_IS_BOUNDARY1D: return m->isB1 ? m->nSurf : 0;
    case OR_A_IS_FEATURE: return m->isFeat ? m->nSurf : 0;
    case OR_A_IS_BOUNDARY2D: return m->isB2 ? m->nV : 0;
    case OR_A_FACE_NORMALS: return m->fn ? 3L * m->nTris : 0;
    case OR_A_VERTEX_NORMALS: return m->vn ? 3L * m->nSurf : 0;
    default: return -1;
    }
}

int or_mesh_array(const or_mesh* m, int id, void* out) {
    long n = or_mesh_array_len(m, id);
    if (n < 0) return -1;
    const void* src = NULL; size_t es = 4;
    switch (id) {
    case OR_A_XYZ: src = m->xyz; break;
    case OR_A_NEW_OF_OLD: src = m->new_of_old; break;
    case OR_A_ELEMS: src = m->elems; break;
    case OR_A_SURF_TRIS: src = m->tris; break;
    case OR_A_HE_ROWPTR: src = m->he_rowptr; break;
    case OR_A_HALFEDGES: src = m->he; break;
    case OR_A_HF_ROWPTR: src = m->hf_rowptr; break;
    case OR_A_HALFFACES: src = m->hf; break;
    case OR_A_COL_FREE: src = m->col_free; break;
    case OR_A_COL_FEATURE: src = m->col_feature; break;
    case OR_A_COL_INNER: src = m->col_inner; break;
    case OR_A_IS_BOUNDARY1D: src = m->isB1; es = 1; break;
    case OR_A_IS_FEATURE: src = m->isFeat; es = 1; break;
    case OR_A_IS_BOUNDARY2D: src = m->isB2; es = 1; break;
    case OR_A_FACE_NORMALS: src = m->fn; break;
    case OR_A_VERTEX_NORMALS: src = m->vn; break;
    }
    if (n > 0 && src) memcpy(out, src, (size_t)n * es);
    return 0;
}

/* accessors used by or_dmo.c */
const int* or__hf_rowptr(const or_mesh* m) { return m->hf_rowptr; }
const int* or__hf(const or_mesh* m) { return m->hf; }
const int* or__he_rowptr(const or_mesh* m) { return m->he_rowptr; }
const int* or__he(const or_mesh* m) { return m->he; }
const int* or__elems(const or_mesh* m) { return m->elems; }
const int* or__col(const or_mesh* m, int which) { return which == 0 ? m->col_free : which == 1 ? m->col_feature : m->col_inner; }
const int* or__faces(const or_mesh* m) { return m->tris; }
int or__fk(const or_mesh* m) { return m->fk; }
const float* or__vn(const or_mesh* m) { return m->vn; }
const float* or__fn(const or_mesh* m) { return m->fn; }
const uint8_t* or__isFeat(const or_mesh* m) { return m->isFeat; }
const uint8_t* or__isB1(const or_mesh* m) { return m->isB1; }
int or__type(const or_mesh* m) { return m->type; }
