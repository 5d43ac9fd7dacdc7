/* CPU oracle for the apspie B200 library -- TEST INFRASTRUCTURE ONLY (see oracle.c). */
#ifndef APSPIE_ORACLE_H
#define APSPIE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

int oracle_bfs(int m, const int *rp, const int *ci, int src, int stop, int *depth);
int oracle_sssp(int m, const int *rp, const int *ci, const int *w, int src, int *dist);
void oracle_mis_greedy(int m, const int *rp, const int *ci, const unsigned *prio,
                       unsigned char *member);
void oracle_mis_vertex_order(int m, const int *rp, const int *ci, int src, int *out);
long long oracle_mis_check(int m, const int *rp, const int *ci, const unsigned char *member);
long long oracle_spgemm_row_nnz(int m, int n, const int *arp, const int *aci, const int *brp,
                                const int *bci, int *crp);
void oracle_spgemm_fill(int m, int n, int vt, const int *arp, const int *aci, const void *aval,
                        const int *brp, const int *bci, const void *bval, const int *crp, int *cci,
                        void *cval);
long long oracle_tc(int m, const int *rp, const int *ci);
void oracle_mt19937(unsigned seed, long long count, unsigned *out);
int oracle_spmspv(int m, int n, int vt, const int *rp, const int *ci, const void *aval, int nx, const int *x_ind,
                  const void *x_val, int *y_ind, void *y_val);

#ifdef __cplusplus
}
#endif

#endif
