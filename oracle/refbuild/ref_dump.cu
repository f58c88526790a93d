// ref_dump.cu -- runs kadircs/hmglib's own GPU build on a given point set and dumps
// what the parity tests compare against.  Linked against the reference's sources by
// oracle/refbuild/build_ref.sh; never part of the product.  TEST INFRASTRUCTURE ONLY.
//
// usage: ref_dump <input.bin> <output.bin>
// input (little endian): int32 n1, n2, dim, bits, c_leaf, k, kernel_type (1 gaussian,
//   2 matern), max_level, precompute_dense, n_apply; float64 eta; then set 1 coords
//   (dim x n1, SoA), set 2 coords (dim x n2), x (n2).
// output: int32 n1, n2, dense_count, aca_count; uint64 codes1[n1], codes2[n2],
//   order1[n1], order2[n2]; int32 blocks[count][5] (set1_l, set1_u, set2_l, set2_u,
//   work_type); float64 y_h[n1] (apply_h_matrix_mvp), y_full[n1] (apply_full_mvp);
//   float64 timings_ms[5]: setup, precompute_aca, precompute_dense, apply (median),
//   apply_full; float64 y_h2[n1]: the product after a second precompute_aca.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hmglib.h"
#include "kernel_system_assembler.h"

static float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

int main(int argc, char** argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s <input.bin> <output.bin>\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[1], "rb");
    if (!f) { perror("input"); return 2; }
    int hdr[10];
    double eta;
    if (fread(hdr, sizeof(int), 10, f) != 10 || fread(&eta, sizeof(double), 1, f) != 1) return 2;
    int n1 = hdr[0], n2 = hdr[1], dim = hdr[2], bits = hdr[3], c_leaf = hdr[4], k = hdr[5];
    int kernel_type = hdr[6], max_level = hdr[7], pre_dense = hdr[8], n_apply = hdr[9];
    std::vector<double> c1((size_t)dim * n1), c2((size_t)dim * n2), x(n2);
    if (fread(c1.data(), sizeof(double), c1.size(), f) != c1.size() ||
        fread(c2.data(), sizeof(double), c2.size(), f) != c2.size() ||
        fread(x.data(), sizeof(double), x.size(), f) != x.size())
        return 2;
    fclose(f);

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double t[5] = {0, 0, 0, 0, 0};

    int pc[2] = {n1, n2};
    struct h_matrix_data data;
    init_h_matrix_data(&data, pc, dim, bits);
    data.eta = eta;
    data.max_level = max_level;
    data.c_leaf = c_leaf;
    data.k = k;
    data.epsilon = 1e-10;
    data.max_batched_dense_size = 1 << 27;
    data.max_batched_aca_size = 1 << 25;
    data.dense_batching_ratio = 0.5;
    data.root_level_set_1 = 0;
    data.root_level_set_2 = 0;
    for (int d = 0; d < dim; d++) {
        cudaMemcpy(data.coords_d[0][d], c1.data() + (size_t)d * n1, sizeof(double) * n1, cudaMemcpyHostToDevice);
        cudaMemcpy(data.coords_d[1][d], c2.data() + (size_t)d * n2, sizeof(double) * n2, cudaMemcpyHostToDevice);
    }
    cudaDeviceSynchronize();

    cudaEventRecord(e0);
    setup_h_matrix(&data);
    cudaEventRecord(e1);
    t[0] = elapsed(e0, e1);

    std::vector<uint64_t> codes1(n1), codes2(n2), ord1(n1), ord2(n2);
    cudaMemcpy(codes1.data(), data.code_d[0], sizeof(uint64_t) * n1, cudaMemcpyDeviceToHost);
    cudaMemcpy(codes2.data(), data.code_d[1], sizeof(uint64_t) * n2, cudaMemcpyDeviceToHost);
    cudaMemcpy(ord1.data(), data.order[0], sizeof(uint64_t) * n1, cudaMemcpyDeviceToHost);
    cudaMemcpy(ord2.data(), data.order[1], sizeof(uint64_t) * n2, cudaMemcpyDeviceToHost);
    int nb = data.mat_vec_data_count;
    std::vector<struct work_item> items(nb);
    cudaMemcpy(items.data(), *data.mat_vec_data, sizeof(struct work_item) * nb, cudaMemcpyDeviceToHost);

    struct system_assembler* assem = nullptr;
    void** slot = nullptr;
    cudaMalloc((void**)&slot, sizeof(void*));
    if (kernel_type == 2)
        create_matern_kernel_system_assembler_object((struct matern_kernel_system_assembler**)slot, 0.0);
    else
        create_gaussian_kernel_system_assembler_object((struct gaussian_kernel_system_assembler**)slot, 0.0);
    cudaMemcpy(&assem, slot, sizeof(void*), cudaMemcpyDeviceToHost);
    data.assem = assem;

    cudaEventRecord(e0);
    precompute_aca(&data);
    cudaEventRecord(e1);
    t[1] = elapsed(e0, e1);
    if (pre_dense) {
        cudaEventRecord(e0);
        precompute_dense(&data);
        cudaEventRecord(e1);
        t[2] = elapsed(e0, e1);
    }

    double *dx = nullptr, *dy = nullptr, *dyf = nullptr;
    cudaMalloc((void**)&dx, sizeof(double) * n2);
    cudaMalloc((void**)&dy, sizeof(double) * n1);
    cudaMalloc((void**)&dyf, sizeof(double) * n1);
    std::vector<float> at;
    for (int a = 0; a < std::max(1, n_apply); a++) {
        cudaMemcpy(dx, x.data(), sizeof(double) * n2, cudaMemcpyHostToDevice);
        cudaMemset(dy, 0, sizeof(double) * n1);
        cudaDeviceSynchronize();
        cudaEventRecord(e0);
        apply_h_matrix_mvp(dx, dy, &data);
        cudaEventRecord(e1);
        at.push_back(elapsed(e0, e1));
    }
    std::sort(at.begin(), at.end());
    t[3] = at[at.size() / 2];
    std::vector<double> yh(n1), yf(n1);
    cudaMemcpy(yh.data(), dy, sizeof(double) * n1, cudaMemcpyDeviceToHost);
    cudaMemcpy(dx, x.data(), sizeof(double) * n2, cudaMemcpyHostToDevice);
    cudaEventRecord(e0);
    apply_full_mvp(dx, dyf, &data);
    cudaEventRecord(e1);
    t[4] = elapsed(e0, e1);
    cudaMemcpy(yf.data(), dyf, sizeof(double) * n1, cudaMemcpyDeviceToHost);
    // a second, independent ACA of the same H-matrix and product: shows the
    // run-to-run variation of the reference's own result
    cudaFree(data.U);
    cudaFree(data.V);
    data.U = data.V = 0;
    precompute_aca(&data);
    cudaMemcpy(dx, x.data(), sizeof(double) * n2, cudaMemcpyHostToDevice);
    cudaMemset(dy, 0, sizeof(double) * n1);
    apply_h_matrix_mvp(dx, dy, &data);
    std::vector<double> yh2(n1);
    cudaMemcpy(yh2.data(), dy, sizeof(double) * n1, cudaMemcpyDeviceToHost);
    cudaError_t err = cudaGetLastError();

    FILE* o = fopen(argv[2], "wb");
    if (!o) { perror("output"); return 2; }
    int oh[4] = {n1, n2, data.mat_vec_info.dense_count, data.mat_vec_info.aca_count};
    fwrite(oh, sizeof(int), 4, o);
    fwrite(codes1.data(), 8, n1, o);
    fwrite(codes2.data(), 8, n2, o);
    fwrite(ord1.data(), 8, n1, o);
    fwrite(ord2.data(), 8, n2, o);
    for (int b = 0; b < nb; b++) {
        int r[5] = {items[b].set1_l, items[b].set1_u, items[b].set2_l, items[b].set2_u, items[b].work_type};
        fwrite(r, sizeof(int), 5, o);
    }
    fwrite(yh.data(), 8, n1, o);
    fwrite(yf.data(), 8, n1, o);
    fwrite(t, 8, 5, o);
    fwrite(yh2.data(), 8, n1, o);
    fclose(o);
    printf("{\"n1\": %d, \"n2\": %d, \"blocks\": %d, \"dense\": %d, \"aca\": %d, \"setup_ms\": %.3f, "
           "\"precompute_aca_ms\": %.3f, \"precompute_dense_ms\": %.3f, \"apply_ms\": %.3f, "
           "\"apply_full_ms\": %.3f, \"cuda\": \"%s\"}\n",
           n1, n2, nb, oh[2], oh[3], t[0], t[1], t[2], t[3], t[4], cudaGetErrorString(err));
    return err == cudaSuccess ? 0 : 1;
}
