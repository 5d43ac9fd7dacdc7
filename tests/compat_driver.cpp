// Test driver for include/apspie/compat.hpp: a program written against the reference's
// entry points (names, argument orders, d_matrix) running on libapspie.so.
//   compat_driver <outdir>
// Builds R-MAT scale 12 (seed 1, weights seed 3) with the library's host generator, loads
// it through matrix_new/buildMatrix from COO, runs bfs<int>, spmspvBfs, sssp<int>,
// sssp<float>, spmspvMis<float>, spmspvCsr, spgemm(d_matrix*), mXm, mXv and triangleCount, and writes
// each result as a raw binary file for the test to compare with the oracle.
#include <cstdio>
#include <string>
#include <vector>

#include "apspie/compat.hpp"

static void dump(const std::string &path, const void *d_ptr, size_t bytes) {
    std::vector<char> h(bytes);
    cudaMemcpy(h.data(), d_ptr, bytes, cudaMemcpyDeviceToHost);
    FILE *f = std::fopen(path.c_str(), "wb");
    std::fwrite(h.data(), 1, bytes, f);
    std::fclose(f);
}

int main(int argc, char **argv) {
    if (argc != 2) return 2;
    const std::string out = argv[1];
    apspie_host_csr g;
    if (apspie_gen_rmat(12, 16, 1, 3, 0.57, 0.19, 0.19, 1, &g) != APSPIE_OK) return 3;
    const int m = g.m, edge = g.nnz;
    const int src = apspie_max_degree_vertex(&g);
    // COO in the reference driver's layout, then the reference's container
    std::vector<int> row(edge), col(edge);
    std::vector<float> val(edge);
    for (int i = 0; i < m; ++i)
        for (int e = g.row_ptr[i]; e < g.row_ptr[i + 1]; ++e) {
            row[e] = i;
            col[e] = g.col_ind[e];
            val[e] = static_cast<float>(static_cast<int *>(g.val)[e]);
        }
    d_matrix A;
    matrix_new(&A, m, m);
    buildMatrix<float>(&A, edge, row.data(), col.data(), val.data());
    int *d_wi = nullptr;
    cudaMalloc(&d_wi, edge * sizeof(int));
    cudaMemcpy(d_wi, g.val, edge * sizeof(int), cudaMemcpyHostToDevice);

    mgpu::ContextPtr context = mgpu::CreateCudaDevice(0);
    context->set_symmetric(true);
    int *d_res = nullptr;
    float *d_resf = nullptr;
    cudaMalloc(&d_res, m * sizeof(int));
    cudaMalloc(&d_resf, m * sizeof(float));

    bfs<float>(src, edge, m, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_res, 1000, *context);
    dump(out + "/bfs.i32", d_res, m * sizeof(int));
    spmspvBfs(src, edge, m, A.h_cscColPtr, A.d_cscColPtr, A.d_cscRowInd, d_res, 1000, *context);
    dump(out + "/spmspvbfs.i32", d_res, m * sizeof(int));
    sssp<int>(src, edge, m, d_wi, A.d_cscColPtr, A.d_cscRowInd, d_res, 1000, *context);
    dump(out + "/sssp.i32", d_res, m * sizeof(int));
    sssp<float>(src, edge, m, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_resf, 1000, *context);
    dump(out + "/sssp.f32", d_resf, m * sizeof(float));

    // MIS with float priorities in [0, 1): mt19937(4) outputs scaled
    std::vector<unsigned> pr(m);
    apspie_mt19937_u32(4, m, pr.data());
    std::vector<float> prf(m);
    for (int i = 0; i < m; ++i) prf[i] = static_cast<float>(pr[i] >> 8) / 16777216.0f;
    float *d_pr = nullptr;
    cudaMalloc(&d_pr, m * sizeof(float));
    cudaMemcpy(d_pr, prf.data(), m * sizeof(float), cudaMemcpyHostToDevice);
    spmspvMis<float>(edge, m, A.h_cscColPtr, A.d_cscColPtr, A.d_cscRowInd, d_pr, d_res, 0.01f, *context);
    dump(out + "/mis.i32", d_res, m * sizeof(int));
    int *d_hop = nullptr;
    cudaMalloc(&d_hop, m * sizeof(int));
    spmspvCsr<int>(d_res, edge, m, A.d_cscColPtr, A.d_cscRowInd, d_hop, *context);
    dump(out + "/hop.i32", d_hop, m * sizeof(int));
    FILE *pf = std::fopen((out + "/mis_prio.f32").c_str(), "wb");
    std::fwrite(prf.data(), sizeof(float), m, pf);
    std::fclose(pf);

    d_matrix C;
    matrix_new(&C, m, m);
    spgemm(&C, &A, &A, 0, 0, *context);
    dump(out + "/spgemm_rp.i32", C.d_cscColPtr, (m + 1) * sizeof(int));
    dump(out + "/spgemm_ci.i32", C.d_cscRowInd, static_cast<size_t>(C.nnz) * sizeof(int));
    dump(out + "/spgemm_v.f32", C.d_cscVal, static_cast<size_t>(C.nnz) * sizeof(float));

    // mXm (src/tc.cuh:315) on two different matrices over CSC arrays: A's CSC arrays are
    // the R-MAT's CSR arrays (so A = R^T) and B's are an Erdos-Renyi matrix E's (B = E^T);
    // the CSC of C = A*B is then the CSR of E*R, which the test checks.
    apspie_host_csr er;
    if (apspie_gen_er(m, 8, 9, APSPIE_VAL_F32, &er) != APSPIE_OK) return 4;
    int *d_erp = nullptr, *d_eci = nullptr;
    float *d_ev = nullptr;
    cudaMalloc(&d_erp, (m + 1) * sizeof(int));
    cudaMalloc(&d_eci, er.nnz * sizeof(int));
    cudaMalloc(&d_ev, er.nnz * sizeof(float));
    cudaMemcpy(d_erp, er.row_ptr, (m + 1) * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(d_eci, er.col_ind, er.nnz * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(d_ev, er.val, er.nnz * sizeof(float), cudaMemcpyHostToDevice);
    const size_t cap = static_cast<size_t>(er.nnz) * 64;  // >= products of E*R
    int *d_cp = nullptr, *d_cr = nullptr;
    float *d_cv = nullptr;
    cudaMalloc(&d_cp, (m + 1) * sizeof(int));
    cudaMalloc(&d_cr, cap * sizeof(int));
    cudaMalloc(&d_cv, cap * sizeof(float));
    const int nnz_c = mXm<float>(edge, m, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_ev, er.row_ptr, d_erp, d_eci,
                                 d_cv, d_cp, d_cr, *context);
    dump(out + "/mxm_rp.i32", d_cp, (m + 1) * sizeof(int));
    dump(out + "/mxm_ci.i32", d_cr, static_cast<size_t>(nnz_c) * sizeof(int));
    dump(out + "/mxm_v.f32", d_cv, static_cast<size_t>(nnz_c) * sizeof(float));
    cudaFree(d_erp);
    cudaFree(d_eci);
    cudaFree(d_ev);
    cudaFree(d_cp);
    cudaFree(d_cr);
    cudaFree(d_cv);

    // mXv (src/mXv.cuh:249): a sparse vector of 64 entries (indices 7 * k mod m, values
    // 0.5 + k / 64, index 0 twice) times A, through the reference's scratch block
    {
        std::vector<int> xi(64);
        std::vector<float> xv(64);
        for (int k = 0; k < 64; ++k) {
            xi[k] = (7 * k) % m;
            xv[k] = 0.5f + k / 64.0f;
        }
        xi[63] = 0;
        int *d_xi = nullptr, *d_yi = nullptr;
        float *d_xv = nullptr, *d_yv = nullptr;
        cudaMalloc(&d_xi, 64 * sizeof(int));
        cudaMalloc(&d_xv, 64 * sizeof(float));
        cudaMalloc(&d_yi, m * sizeof(int));
        cudaMalloc(&d_yv, m * sizeof(float));
        cudaMemcpy(d_xi, xi.data(), 64 * sizeof(int), cudaMemcpyHostToDevice);
        cudaMemcpy(d_xv, xv.data(), 64 * sizeof(float), cudaMemcpyHostToDevice);
        d_scratch *scr = nullptr;
        allocScratch(&scr, edge, m);
        int nnz_y = 64;
        mXv<float>(d_xi, d_xv, edge, m, nnz_y, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_yi, d_yv, scr, *context);
        freeScratch(scr);
        dump(out + "/mxv_i.i32", d_yi, static_cast<size_t>(nnz_y) * sizeof(int));
        dump(out + "/mxv_v.f32", d_yv, static_cast<size_t>(nnz_y) * sizeof(float));
        cudaFree(d_xi);
        cudaFree(d_xv);
        cudaFree(d_yi);
        cudaFree(d_yv);
    }

    long long tri = triangleCount(edge, m, A.d_cscColPtr, A.d_cscRowInd, *context);
    FILE *tf = std::fopen((out + "/tc.txt").c_str(), "w");
    std::fprintf(tf, "%lld\n", tri);
    std::fclose(tf);
    cudaError_t e = cudaDeviceSynchronize();
    std::printf("compat driver done: %s\n", cudaGetErrorString(e));
    matrix_delete(&A);
    matrix_delete(&C);
    apspie_host_csr_free(&g);
    apspie_host_csr_free(&er);
    return e == cudaSuccess ? 0 : 1;
}
