// ref_gpu_labels.cpp -- runs the reference's OWN compiled GPU label phases on given inputs.
//
// TEST INFRASTRUCTURE ONLY.  Linked by oracle/Makefile against the object files of the reference's
// cudaKernel.cu / cudaKernel_gaussian.cu / cudaKernel_multinomial.cu (compiled out-of-tree for
// sm_100a) and its host sources.  It is run as a child process by tests/test_gpu_reference_labels.py,
// because cudaKernel::init calls cudaDeviceReset (cudaKernel.cu:615), which would end the CUDA state of
// the test process.  With fixed cluster parameters and the reference's per-point XORWOW stream
// (initCurand: curand_init(seed, point, 0), cudaKernel.cu:19-25) it produces the labels that
//   cudaKernel::create_clusters_labels      (cudaKernel.cu:1400-1490; softmax + alias, or argmax)
//   cudaKernel::create_subclusters_labels   (cudaKernel.cu:1299-1398)
// draw, for the test to compare point by point with this repository's kernels in cuRAND-compatible
// mode.
//
// usage: ref_gpu_labels <input> <output>
// input (little-endian): int32 prior (0 NIW, 1 multinomial), int32 N, int32 D, int32 K, uint64 seed,
//   points D*N doubles (point n at [n*D, n*D + D)), then per cluster k:
//     NIW:          mu[D], invSigma[D*D] (column-major), logdetSigma  for the cluster, l, r
//     multinomial:  log theta[D]                                       for the cluster, l, r
//   then weight[K], lr_weights[2K]
// output: int32 labels[N] (sampled), int32 sub_labels[N] (sampled, using those labels),
//         int32 labels_final[N] (argmax; no random numbers consumed)
#include <cstdint>
#include <cstdio>
#include <memory>
#include <vector>

#include "cudaKernel_gaussian.cuh"
#include "cudaKernel_multinomial.cuh"
#include "distributions/multinomial_dist.h"
#include "distributions/mv_gaussian.h"

namespace {

template <typename T>
bool rd(FILE* f, T* p, size_t n)
{
    return fread(p, sizeof(T), n, f) == n;
}

std::shared_ptr<distribution_sample> read_dist(FILE* f, int prior, int D, bool* ok)
{
    if (prior == 0) {
        auto g = std::make_shared<mv_gaussian>();
        g->mu.resize(D);
        g->invSigma.resize(D, D);
        g->sigma = Eigen::MatrixXd::Identity(D, D);   // not read by the label phases
        *ok = *ok && rd(f, g->mu.data(), (size_t)D) && rd(f, g->invSigma.data(), (size_t)D * D) &&
              rd(f, &g->logdetSigma, 1);
        return g;
    }
    auto m = std::make_shared<multinomial_dist>();
    m->alpha.resize(D);
    *ok = *ok && rd(f, m->alpha.data(), (size_t)D);
    return m;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[1], "rb");
    if (!f) {
        fprintf(stderr, "cannot open %s\n", argv[1]);
        return 2;
    }
    int32_t hdr[4];
    uint64_t seed = 0;
    bool ok = rd(f, hdr, 4) && rd(f, &seed, 1);
    const int prior = hdr[0], N = hdr[1], D = hdr[2], K = hdr[3];
    if (!ok || N <= 0 || D <= 0 || K <= 0 || (prior != 0 && prior != 1)) {
        fprintf(stderr, "bad header\n");
        return 2;
    }
    Eigen::MatrixXd points(D, N);
    ok = rd(f, points.data(), (size_t)D * N);
    std::vector<std::shared_ptr<thin_cluster_params>> params;
    std::vector<std::shared_ptr<distribution_sample>> dists(3 * (size_t)K);
    for (int k = 0; k < K; ++k)
        for (int s = 0; s < 3; ++s) dists[3 * (size_t)k + s] = read_dist(f, prior, D, &ok);
    std::vector<double> weights(K), lrw(2 * (size_t)K);
    ok = ok && rd(f, weights.data(), (size_t)K) && rd(f, lrw.data(), 2 * (size_t)K);
    fclose(f);
    if (!ok) {
        fprintf(stderr, "short input\n");
        return 2;
    }
    for (int k = 0; k < K; ++k)
        params.push_back(std::make_shared<thin_cluster_params>(
            dists[3 * (size_t)k], dists[3 * (size_t)k + 1], dists[3 * (size_t)k + 2],
            std::vector<double>{lrw[2 * (size_t)k], lrw[2 * (size_t)k + 1]}));

    std::unique_ptr<cudaKernel> ck;
    if (prior == 0) ck.reset(new cudaKernel_gaussian());
    else ck.reset(new cudaKernel_multinomial());
    ck->init(N, points, (unsigned long long)seed, false, 1);

    auto labels = std::make_shared<LabelsType>();
    auto sub = std::make_shared<LabelsType>();
    auto final_labels = std::make_shared<LabelsType>();
    ck->create_clusters_labels(K, params, weights, false);
    ck->get_labels(labels);
    ck->create_subclusters_labels(K, params, D);
    ck->get_sub_labels(sub);
    ck->create_clusters_labels(K, params, weights, true);
    ck->get_labels(final_labels);
    ck->release();

    FILE* o = fopen(argv[2], "wb");
    if (!o) {
        fprintf(stderr, "cannot open %s\n", argv[2]);
        return 2;
    }
    bool w = fwrite(labels->data(), sizeof(int), (size_t)N, o) == (size_t)N &&
             fwrite(sub->data(), sizeof(int), (size_t)N, o) == (size_t)N &&
             fwrite(final_labels->data(), sizeof(int), (size_t)N, o) == (size_t)N;
    fclose(o);
    return w ? 0 : 2;
}
