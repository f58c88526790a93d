// legacy_driver.cu -- a driver written against the reference's interface only
// (include/hmglib.h, include/kernel_system_assembler.h), following the flow of the
// reference's own test program (hmglib_test.cu:25-142): points written straight
// into data.coords_d, setup, Gaussian assembler through a device slot,
// precompute_aca (+ precompute_dense), apply_full_mvp, apply_h_matrix_mvp, relative
// error.  Points come from SplitMix64 instead of cuRAND so the result is
// reproducible.  Prints one JSON line; exit status 0 when the error is below the
// bound given on the command line.
//
// usage: legacy_driver <N> <k> <c_leaf> <eta> <precompute_dense 0|1> <max_rel_err>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hmglib.h"
#include "kernel_system_assembler.h"

static uint64_t splitmix(uint64_t seed, uint64_t i)
{
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double unif(uint64_t seed, uint64_t i) { return (double)(splitmix(seed, i) >> 11) * (1.0 / 9007199254740992.0); }

int main(int argc, char** argv)
{
    if (argc != 7) {
        printf("%s <N> <k> <c_leaf> <eta> <precompute_dense> <max_rel_err>\n", argv[0]);
        return 2;
    }
    const int dim = 2, bits = 32;
    int point_count[2];
    point_count[0] = point_count[1] = atoi(argv[1]);
    const int n = point_count[0];

    struct h_matrix_data data;
    init_h_matrix_data(&data, point_count, dim, bits);
    data.eta = atof(argv[4]);
    data.max_level = 50;
    data.c_leaf = atoi(argv[3]);
    data.k = atoi(argv[2]);
    data.epsilon = 1e-10;
    data.max_batched_dense_size = 8192;
    data.max_batched_aca_size = 65536;
    data.root_level_set_1 = 0;
    data.root_level_set_2 = 0;

    // points: uniform in [0,1]^2 scaled by 1/sqrt(0.1) (exp(-r^2/0.1)), point-major
    std::vector<double> c((size_t)dim * n);
    const double s = 1.0 / std::sqrt(0.1);
    for (int i = 0; i < n; i++)
        for (int d = 0; d < dim; d++) c[(size_t)d * n + i] = unif(0, (uint64_t)i * dim + d) * s;
    for (int d = 0; d < dim; d++) {
        cudaMemcpy(data.coords_d[0][d], c.data() + (size_t)d * n, sizeof(double) * n, cudaMemcpyHostToDevice);
        cudaMemcpy(data.coords_d[1][d], c.data() + (size_t)d * n, sizeof(double) * n, cudaMemcpyHostToDevice);
    }

    setup_h_matrix(&data);

    struct gaussian_kernel_system_assembler** assem_d_p;
    cudaMalloc((void***)&assem_d_p, sizeof(struct gaussian_kernel_system_assembler*));
    create_gaussian_kernel_system_assembler_object(assem_d_p, 0.0);
    struct gaussian_kernel_system_assembler* assem_d;
    cudaMemcpy(&assem_d, assem_d_p, sizeof(struct gaussian_kernel_system_assembler*), cudaMemcpyDeviceToHost);
    data.assem = assem_d;

    precompute_aca(&data);
    if (atoi(argv[5])) precompute_dense(&data);

    std::vector<double> xh(n);
    for (int i = 0; i < n; i++) xh[i] = 2.0 * unif(1000, i) - 1.0;
    double *x, *y, *y_test;
    cudaMalloc((void**)&x, sizeof(double) * n);
    cudaMalloc((void**)&y, sizeof(double) * n);
    cudaMalloc((void**)&y_test, sizeof(double) * n);
    cudaMemcpy(x, xh.data(), sizeof(double) * n, cudaMemcpyHostToDevice);

    apply_full_mvp(x, y_test, &data);
    apply_h_matrix_mvp(x, y, &data);

    std::vector<double> a(n), b(n), x2(n);
    cudaMemcpy(a.data(), y, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(b.data(), y_test, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(x2.data(), x, sizeof(double) * n, cudaMemcpyDeviceToHost);
    double num = 0, den = 0;
    bool x_same = true;
    for (int i = 0; i < n; i++) {
        num += (a[i] - b[i]) * (a[i] - b[i]);
        den += b[i] * b[i];
        x_same = x_same && x2[i] == xh[i];
    }
    double err = std::sqrt(num / den);

    // the sorted codes and the permutation are visible like in the reference
    std::vector<uint64_t> codes(n), order(n);
    cudaMemcpy(codes.data(), data.code_d[0], sizeof(uint64_t) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(order.data(), data.order[0], sizeof(uint64_t) * n, cudaMemcpyDeviceToHost);
    bool sorted = true, perm_ok = true;
    std::vector<char> seen(n, 0);
    for (int i = 0; i < n; i++) {
        if (i && codes[i] < codes[i - 1]) sorted = false;
        if (order[i] >= (uint64_t)n || seen[order[i]]) perm_ok = false; else seen[order[i]] = 1;
    }

    printf("{\"n\": %d, \"blocks\": %d, \"dense\": %d, \"aca\": %d, \"rel_err\": %.6e, \"x_unchanged\": %d, "
           "\"codes_sorted\": %d, \"order_is_permutation\": %d}\n",
           n, data.mat_vec_data_count, data.mat_vec_info.dense_count, data.mat_vec_info.aca_count, err,
           (int)x_same, (int)sorted, (int)perm_ok);

    cudaFree(x);
    cudaFree(y);
    cudaFree(y_test);
    destroy_gaussian_kernel_system_assembler_object(assem_d_p);
    cudaFree(assem_d_p);
    destroy_h_matrix_data(&data);
    bool ok = err < atof(argv[6]) && x_same && sorted && perm_ok && cudaGetLastError() == cudaSuccess;
    return ok ? 0 : 1;
}
