/*
 * CPU oracle for the apspie B200 library -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatements of the reference's algorithms on the SpMSpV / SpGEMM hot path,
 * used by tests/ (as the checker), by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg. The product never links, loads or calls anything here.
 *
 * Pinning: BFS and SSSP are cross-checked against the reference's own CPU code compiled
 * from its sources into oracle/_ref (bfsCPU src/testBfs.cpp:75, ssspCPU
 * src/testSssp.cpp:117) and against golden vectors made from it (tests/golden). MIS,
 * SpGEMM and TC have no CPU implementation or stored answers in the reference
 * (test/tc/main.cu:220 prints an unchecked count); those restatements are pinned only by
 * the reference's property checks (MIS: src/util.cuh:271-316 unverify) and by
 * independent brute-force cross-checks in tests/ -- parity unpinned by reference outputs.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

/* ---- BFS: queue BFS of SimpleReferenceBfs (src/testBfs.cpp:6-72) ---------------- */
int oracle_bfs(int m, const int *rp, const int *ci, int src, int stop, int *depth) {
    int *queue = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    int head = 0, tail = 0, search_depth = 0;
    for (int i = 0; i < m; ++i) depth[i] = -1;
    depth[src] = 0;
    queue[tail++] = src;
    while (head < tail) {
        int v = queue[head++];
        int nd = depth[v] + 1;
        if (nd > stop) break; /* testBfs.cpp:40-41 */
        for (int e = rp[v]; e < rp[v + 1]; ++e) {
            int u = ci[e];
            if (depth[u] == -1) {
                depth[u] = nd;
                if (search_depth < nd) search_depth = nd;
                queue[tail++] = u;
            }
        }
    }
    free(queue);
    return search_depth + 1; /* testBfs.cpp:65 */
}

/* ---- SSSP: label-correcting priority-queue search of SimpleReferenceSssp
 *      (src/testSssp.cpp:33-115) with int32 weights and int64 path sums ------------- */
typedef struct { long long d; int v; } heap_item;

static void heap_push(heap_item *h, long long *n, heap_item x) {
    long long i = (*n)++;
    while (i > 0) {
        long long p = (i - 1) / 2;
        if (h[p].d <= x.d) break;
        h[i] = h[p];
        i = p;
    }
    h[i] = x;
}

static heap_item heap_pop(heap_item *h, long long *n) {
    heap_item top = h[0], x = h[--(*n)];
    long long i = 0;
    for (;;) {
        long long l = 2 * i + 1, r = l + 1, s = i;
        long long best_d = x.d;
        if (l < *n && h[l].d < best_d) { s = l; best_d = h[l].d; }
        if (r < *n && h[r].d < best_d) { s = r; }
        if (s == i) break;
        h[i] = h[s];
        i = s;
    }
    h[i] = x;
    return top;
}

int oracle_sssp(int m, const int *rp, const int *ci, const int *w, int src, int *dist) {
    long long nnz = rp[m];
    long long cap = nnz + m + 1, n = 0;
    heap_item *h = (heap_item *)malloc(sizeof(heap_item) * (size_t)cap);
    long long *d = (long long *)malloc(sizeof(long long) * (size_t)(m > 0 ? m : 1));
    int rc = 0;
    for (int i = 0; i < m; ++i) d[i] = -1;
    d[src] = 0;
    heap_item s0 = {0, src};
    heap_push(h, &n, s0);
    while (n > 0) {
        heap_item t = heap_pop(h, &n);
        if (t.d != d[t.v]) continue; /* stale entry: only the best copy relaxes */
        for (int e = rp[t.v]; e < rp[t.v + 1]; ++e) {
            int u = ci[e];
            if (w[e] < 0) { rc = -2; continue; }
            long long alt = t.d + w[e];
            if (d[u] == -1 || alt < d[u]) {
                d[u] = alt;
                if (n < cap) {
                    heap_item it = {alt, u};
                    heap_push(h, &n, it);
                } else {
                    rc = -3;
                }
            }
        }
    }
    for (int i = 0; i < m; ++i) {
        if (d[i] > 2147483646LL) rc = -1;
        dist[i] = (int)d[i];
    }
    free(h);
    free(d);
    return rc;
}

/* ---- MIS ---------------------------------------------------------------------- */

/* Greedy MIS in descending (priority, id) order: the fixed point of spmspvMis's
 * priority-thresholded Luby rounds (src/spmspvMis.cuh:54-78, 232-318): a vertex is
 * selected exactly when it outranks every still-undecided neighbour, and selected
 * vertices knock their neighbours out. Self-loops are ignored. */
static const unsigned *g_prio;
static int cmp_desc(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    if (g_prio[x] != g_prio[y]) return g_prio[x] > g_prio[y] ? -1 : 1;
    return x > y ? -1 : (x < y ? 1 : 0);
}

void oracle_mis_greedy(int m, const int *rp, const int *ci, const unsigned *prio,
                       unsigned char *member) {
    int *order = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    unsigned char *out = (unsigned char *)calloc((size_t)(m > 0 ? m : 1), 1);
    for (int i = 0; i < m; ++i) order[i] = i;
    g_prio = prio;
    qsort(order, (size_t)m, sizeof(int), cmp_desc);
    for (int i = 0; i < m; ++i) member[i] = 0;
    for (int k = 0; k < m; ++k) {
        int v = order[k];
        if (out[v]) continue;
        member[v] = 1;
        for (int e = rp[v]; e < rp[v + 1]; ++e)
            if (ci[e] != v) out[ci[e]] = 1;
    }
    free(order);
    free(out);
}

/* Vertex-order greedy MIS of SimpleReferenceMis (test/mis/main.cu:25-88): `src` first,
 * then every still-undecided vertex in id order. out[i] in {1, 0}. */
void oracle_mis_vertex_order(int m, const int *rp, const int *ci, int src, int *out) {
    for (int i = 0; i < m; ++i) out[i] = -1;
    out[src] = 1;
    for (int e = rp[src]; e < rp[src + 1]; ++e)
        if (out[ci[e]] == -1) out[ci[e]] = 0;
    for (int i = 0; i < m; ++i) {
        if (out[i] != -1) continue;
        out[i] = 1;
        for (int e = rp[i]; e < rp[i + 1]; ++e)
            if (out[ci[e]] == -1) out[ci[e]] = 0;
    }
}

/* The reference's MIS validity check: y = one-hop of the set (spmspvCsr,
 * src/spmspvMis.cuh:81-147) and then member[i] + y[i] == 1 for all i
 * (uncompareResults, src/util.cuh:271-303). Returns the number of violations. */
long long oracle_mis_check(int m, const int *rp, const int *ci, const unsigned char *member) {
    int *y = (int *)calloc((size_t)(m > 0 ? m : 1), sizeof(int));
    long long bad = 0;
    for (int v = 0; v < m; ++v)
        if (member[v])
            for (int e = rp[v]; e < rp[v + 1]; ++e) y[ci[e]] = 1;
    for (int i = 0; i < m; ++i)
        if ((int)member[i] + y[i] != 1) ++bad;
    free(y);
    return bad;
}

/* ---- SpGEMM: row-wise Gustavson with a dense accumulator ------------------------
 * C = A*B; each output row's entries are summed in increasing position of A's row
 * (k order), products and sums rounded separately (no fused multiply-add), columns
 * sorted. This is the result of the reference's hash SpGEMM (spgemmKernel.cuh:211-343)
 * up to summation order, which the reference leaves to atomicAdd. */
long long oracle_spgemm_row_nnz(int m, int n, const int *arp, const int *aci, const int *brp,
                                const int *bci, int *crp) {
    int *mark = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    long long total = 0;
    for (int j = 0; j < n; ++j) mark[j] = -1;
    crp[0] = 0;
    for (int i = 0; i < m; ++i) {
        int cnt = 0;
        for (int ea = arp[i]; ea < arp[i + 1]; ++ea) {
            int k = aci[ea];
            for (int eb = brp[k]; eb < brp[k + 1]; ++eb) {
                int j = bci[eb];
                if (mark[j] != i) { mark[j] = i; ++cnt; }
            }
        }
        total += cnt;
        crp[i + 1] = (int)total;
    }
    free(mark);
    return total;
}

static int cmp_int(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* vt: 1 = float, 2 = int32 (apspie_val_type) */
void oracle_spgemm_fill(int m, int n, int vt, const int *arp, const int *aci, const void *aval,
                        const int *brp, const int *bci, const void *bval, const int *crp, int *cci,
                        void *cval) {
    int *mark = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    float *accf = (float *)calloc((size_t)(n > 0 ? n : 1), sizeof(float));
    int *acci = (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int));
    for (int j = 0; j < n; ++j) mark[j] = -1;
    for (int i = 0; i < m; ++i) {
        int p = crp[i];
        for (int ea = arp[i]; ea < arp[i + 1]; ++ea) {
            int k = aci[ea];
            for (int eb = brp[k]; eb < brp[k + 1]; ++eb) {
                int j = bci[eb];
                if (mark[j] != i) {
                    mark[j] = i;
                    cci[p++] = j;
                    accf[j] = 0.0f;
                    acci[j] = 0;
                }
                if (vt == 1) {
                    volatile float prod = ((const float *)aval)[ea] * ((const float *)bval)[eb];
                    volatile float sum = accf[j] + prod;
                    accf[j] = sum;
                } else if (vt == 2) {
                    acci[j] += ((const int *)aval)[ea] * ((const int *)bval)[eb];
                }
            }
        }
        qsort(cci + crp[i], (size_t)(p - crp[i]), sizeof(int), cmp_int);
        for (int q = crp[i]; q < p; ++q) {
            if (vt == 1) ((float *)cval)[q] = accf[cci[q]];
            else if (vt == 2) ((int *)cval)[q] = acci[cci[q]];
        }
    }
    free(mark);
    free(accf);
    free(acci);
}

/* ---- TC: sum over L of |L(i,:) n L(k,:)| by sorted merge (int64) --------------------
 * Equals sum((L*L) .* L) for the strict lower triangle L, which is the count the
 * reference obtains as sum((U*L) .* U) with cuSPARSE + ewiseMultTc on CSC arrays
 * (test/tc/main.cu:243-249, src/tc.cuh:168-199). Rows of L must be sorted. */
long long oracle_tc(int m, const int *rp, const int *ci) {
    long long count = 0;
    for (int i = 0; i < m; ++i) {
        for (int e = rp[i]; e < rp[i + 1]; ++e) {
            int k = ci[e];
            int a = rp[i], ae = rp[i + 1], b = rp[k], be = rp[k + 1];
            while (a < ae && b < be) {
                int x = ci[a], y = ci[b];
                if (x == y) { ++count; ++a; ++b; }
                else if (x < y) ++a;
                else ++b;
            }
        }
    }
    return count;
}

/* ---- MT19937 (Matsumoto & Nishimura 1998, 32-bit): the generator behind the
 *      reference's init_genrand/genrand_int32 (src/mt19937ar.cpp:57,102) ------------ */
void oracle_mt19937(unsigned seed, long long count, unsigned *out) {
    unsigned mt[624];
    int idx = 624;
    mt[0] = seed;
    for (int i = 1; i < 624; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (unsigned)i;
    for (long long c = 0; c < count; ++c) {
        if (idx >= 624) {
            for (int i = 0; i < 624; ++i) {
                unsigned y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
                mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
            }
            idx = 0;
        }
        unsigned y = mt[idx++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        out[c] = y;
    }
}

/* Sparse vector times matrix, y = x^T A (the reference's mXv<T>, src/mXv.cuh:249-389:
 * gather the vector's rows, multiply, sort by column, sum runs of equal columns). Each
 * column's sum runs in x's entry order, then row order, starting from 0. vt 1: f32 (no
 * contraction: this file is built with -ffp-contract=off), 2: int32 (wrapping). Writes the
 * touched columns ascending into y_ind / y_val and returns their number. */
int oracle_spmspv(int m, int n, int vt, const int *rp, const int *ci, const void *aval, int nx, const int *x_ind,
                  const void *x_val, int *y_ind, void *y_val) {
    unsigned char *hit = (unsigned char *)calloc((size_t)(n > 0 ? n : 1), 1);
    float *accf = (float *)calloc((size_t)(n > 0 ? n : 1), sizeof(float));
    unsigned *acci = (unsigned *)calloc((size_t)(n > 0 ? n : 1), sizeof(unsigned));
    (void)m;
    for (int j = 0; j < nx; ++j) {
        const int r = x_ind[j];
        for (int e = rp[r]; e < rp[r + 1]; ++e) {
            const int c = ci[e];
            hit[c] = 1;
            if (vt == 1) {
                const float p = ((const float *)x_val)[j] * ((const float *)aval)[e];
                accf[c] = accf[c] + p;
            } else {
                acci[c] += ((const unsigned *)x_val)[j] * ((const unsigned *)aval)[e];
            }
        }
    }
    int k = 0;
    for (int c = 0; c < n; ++c)
        if (hit[c]) {
            y_ind[k] = c;
            if (vt == 1)
                ((float *)y_val)[k] = accf[c];
            else
                ((unsigned *)y_val)[k] = acci[c];
            ++k;
        }
    free(hit);
    free(accf);
    free(acci);
    return k;
}
