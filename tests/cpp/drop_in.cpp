// A caller written against the reference's own API, the way its examples use
// it (examples/miniExample.cpp:102-116, examples/threadedExample.cpp:44-113):
// build an object, turn it into a Fourier modulus with diffractionIntensity,
// reconstruct it with cudaShrinkWrap, then run a batch through the task
// queue; then the fixed-support HIO (libs::hybridInputOutput) and the device
// reductions of algorithms/cuda/cudaVectorReduce.hpp on buffers the caller
// allocates.  Compiled against include/imresh (the reference's header paths)
// and linked against libimresh_b200.so (plus the CUDA runtime for the
// caller's own cudaMalloc).  Prints "OK" on success.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "algorithms/cuda/cudaShrinkWrap.hpp"
#include "algorithms/cuda/cudaVectorReduce.hpp"
#include "libs/hybridInputOutput.hpp"
#include "io/taskQueue.cu"
#include "io/readInFuncs/readInFuncs.hpp"
#include "io/writeOutFuncs/writeOutFuncs.hpp"
#include "libs/diffractionIntensity.hpp"

// a few Gaussian blobs near the centre (deterministic)
static float *make_object(unsigned W, unsigned H)
{
    float *p = new float[W * H];
    std::memset(p, 0, sizeof(float) * W * H);
    const float cx[5] = {0.50f, 0.45f, 0.56f, 0.52f, 0.47f}, cy[5] = {0.50f, 0.54f, 0.47f, 0.58f, 0.44f};
    for (int b = 0; b < 5; ++b)
        for (unsigned y = 0; y < H; ++y)
            for (unsigned x = 0; x < W; ++x) {
                const float dx = x - cx[b] * W, dy = y - cy[b] * H;
                p[y * W + x] += std::exp(-(dx * dx + dy * dy) / 8.f);
            }
    return p;
}

static bool finite(const float *p, size_t n)
{
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

int main()
{
    const unsigned W = 256, H = 192;
    float *pData = make_object(W, H);
    imresh::libs::diffractionIntensity(pData, W, H);
    std::vector<float> modulus(pData, pData + W * H);

    // miniExample's call: 96 blocks x 256 threads (ignored), 64 cycles,
    // target 1e-6, default beta, autocorrelation cutoff 0.001, cutoff 0.01
    int rc = imresh::algorithms::cuda::cudaShrinkWrap(pData, W, H, cudaStream_t(0), 96, 256, 64, 1e-6, 0,
                                                        0.001, 0.01, 0, 0);
    if (rc != 0 || !finite(pData, W * H)) {
        std::printf("cudaShrinkWrap failed: rc=%d\n", rc);
        return 1;
    }
    delete[] pData;

    // threadedExample's pattern: init, N tasks with a write-out callback, deinit
    imresh::io::taskQueueInit();
    std::atomic<int> finished{0}, bad{0};
    const int nTasks = 12;
    for (int i = 0; i < nTasks; ++i) {
        float *task = new float[W * H];
        std::memcpy(task, modulus.data(), sizeof(float) * W * H);
        imresh::io::addTask(task, W, H,
                            [&](float *mem, unsigned const w, unsigned const h, std::string name) {
                                if (w != W || h != H || !finite(mem, (size_t)w * h) || name.empty()) ++bad;
                                ++finished;
                                imresh::io::writeOutFuncs::justFree(mem, w, h, name);
                            },
                            "task_" + std::to_string(i), 4 + i % 3 /* cycles */);
    }
    imresh::io::taskQueueDeinit();
    if (finished != nTasks || bad != 0) {
        std::printf("task queue: finished %d of %d, bad %d\n", (int)finished, nTasks, (int)bad);
        return 1;
    }
    // hybridInputOutput: fixed disk support, 30 iterations, no error test
    std::vector<float> io(modulus);
    std::vector<uint8_t> mask(W * H);
    for (unsigned y = 0; y < H; ++y)
        for (unsigned x = 0; x < W; ++x) {
            const float dx = x - 0.5f * W, dy = y - 0.5f * H;
            mask[y * W + x] = dx * dx + dy * dy > 40.f * 40.f ? 1 : 0;
        }
    rc = imresh::libs::hybridInputOutput(io.data(), mask.data(), std::vector<unsigned>{H, W}, 30, 0.f);
    if (rc != 0 || !finite(io.data(), io.size())) {
        std::printf("hybridInputOutput failed: rc=%d\n", rc);
        return 1;
    }
    if (imresh::libs::hybridInputOutput(io.data(), mask.data(), std::vector<unsigned>{H}, 3) != 1) {
        std::printf("hybridInputOutput accepted a 1D size\n");
        return 1;
    }

    // device reductions: (3, 4) where masked -> total = 5 * count
    const unsigned n = 4096;
    std::vector<float> hz(2 * n), hm(n);
    for (unsigned i = 0; i < n; ++i) {
        hm[i] = (i % 3 == 0) ? 1.f : 0.f;
        hz[2 * i] = hm[i] ? 3.f : 0.25f;
        hz[2 * i + 1] = hm[i] ? 4.f : 0.5f;
    }
    float *dz = nullptr, *dm = nullptr;
    if (cudaMalloc(&dz, sizeof(float) * 2 * n) != cudaSuccess || cudaMalloc(&dm, sizeof(float) * n) != cudaSuccess) {
        std::printf("cudaMalloc failed\n");
        return 1;
    }
    cudaMemcpy(dz, hz.data(), sizeof(float) * 2 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dm, hm.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
    float total = 0, count = 0;
    const float err = imresh::algorithms::cuda::cudaCalculateHioError((const float2 *)dz, (const float *)dm, n,
                                                                      false, cudaStream_t(0), &total, &count);
    const float mx = imresh::algorithms::cuda::cudaVectorMax((const float *)dz, 2 * n);
    cudaFree(dz);
    cudaFree(dm);
    if (count != 1366.f || total != 5.f * count || !(err > 0) || mx != 4.f) {
        std::printf("reductions: count %g total %g err %g max %g\n", count, total, err, mx);
        return 1;
    }
    // file callbacks: a task result written with writeOutNpy / writeOutTxt and read back
    {
        const unsigned w = 5, h = 3;
        float *img = new float[w * h];
        for (unsigned i = 0; i < w * h; ++i) img[i] = 0.25f * i - 1.f;
        const std::string npy = "drop_in_io_test.npy", txt = "drop_in_io_test.txt";
        imresh::io::writeOutFuncs::writeOutNpy(img, w, h, npy);
        imresh::io::writeOutFuncs::writeOutAndFreeTxt(img, w, h, txt);   // releases img
        auto a = imresh::io::readInFuncs::readNpy(npy);
        auto b = imresh::io::readInFuncs::readTxt(txt);
        bool same = a.first && b.first && a.second.first == w && a.second.second == h &&
                    b.second.first == w && b.second.second == h;
        for (unsigned i = 0; same && i < w * h; ++i)
            same = a.first[i] == 0.25f * i - 1.f && b.first[i] == a.first[i];
        imresh::io::writeOutFuncs::justFree(a.first, w, h, npy);
        imresh::io::writeOutFuncs::justFree(b.first, w, h, txt);
        std::remove(npy.c_str());
        std::remove(txt.c_str());
        if (!same) {
            std::printf("file callbacks: read-back mismatch\n");
            return 1;
        }
    }
    std::printf("OK\n");
    return 0;
}
