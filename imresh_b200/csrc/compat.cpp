// The reference's C++ entry points for this path, implemented over the C ABI:
//   imresh::algorithms::cuda::cudaShrinkWrap  -> imr_cuda_shrink_wrap
//   imresh::io::taskQueueInit / addTask / taskQueueDeinit
//                                            -> one imr_engine driven by a
//                                               worker thread, write-out
//                                               callbacks on a second thread
//   imresh::io::writeOutFuncs::justFree       -> delete[]
//   imresh::libs::diffractionIntensity        -> imr_diffraction_intensity
//   imresh::libs::hybridInputOutput           -> imr_hybrid_input_output
#include <cuda_runtime.h>
#include <limits.h>
#include <stdio.h>

#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "imresh_b200.h"
#include "imresh/algorithms/cuda/cudaShrinkWrap.hpp"
#include "imresh/io/taskQueue.hpp"
#include "imresh/io/writeOutFuncs/writeOutFuncs.hpp"
#include "imresh/libs/hybridInputOutput.hpp"

namespace imresh
{
namespace algorithms
{
namespace cuda
{
    int cudaShrinkWrap(float *const rIoData, unsigned int const rImageWidth, unsigned int const rImageHeight,
                       cudaStream_t const rStream, unsigned int rnBlocks, unsigned int rnThreads,
                       unsigned int rnCycles, float rTargetError, float rHioBeta,
                       float rIntensityCutOffAutoCorel, float rIntensityCutOff, float rSigma0,
                       float rSigmaChange, unsigned int rnHioCycles)
    {
        return imr_cuda_shrink_wrap(rIoData, rImageWidth, rImageHeight, (void *)rStream, rnBlocks, rnThreads,
                                    rnCycles, rTargetError, rHioBeta, rIntensityCutOffAutoCorel,
                                    rIntensityCutOff, rSigma0, rSigmaChange, rnHioCycles);
    }
} // namespace cuda
} // namespace algorithms

namespace libs
{
    // diffractionIntensity (src/imresh/libs/diffractionIntensity.hpp, the
    // cuFFT variant's signature): |FFT2(rpIoData)| in place, host buffer.
    void diffractionIntensity(float *const rpIoData, unsigned int const rImageWidth,
                              unsigned int const rImageHeight, cudaStream_t const rStream, bool)
    {
        int rc = imr_diffraction_intensity(rpIoData, rImageWidth, rImageHeight, (void *)rStream);
        if (rc != IMR_SUCCESS)
            fprintf(stderr, "imresh_b200 diffractionIntensity: %s\n", imr_status_string(rc));
    }

    // hybridInputOutput (src/imresh/libs/hybridInputOutput.hpp:81-90): rSize =
    // {rows, columns} as the reference's FFTW plan takes it; 1 for a wrong
    // dimension count or a NULL buffer, as the reference (cpp:199-206).
    int hybridInputOutput(float *const rIoData, uint8_t const *const rMask,
                          std::vector<unsigned int> const rSize, unsigned int rnCycles,
                          float rTargetError, float rBeta, unsigned int)
    {
        if (rSize.size() != 2 || rIoData == NULL || rMask == NULL) return 1;
        return imr_hybrid_input_output(rIoData, rMask, rSize[1], rSize[0],
                                       rnCycles == UINT_MAX ? 0u : rnCycles, rTargetError, rBeta,
                                       nullptr);
    }
} // namespace libs

namespace io
{
namespace writeOutFuncs
{
    void justFree(float *mem, unsigned int const, unsigned int const, std::string const)
    {
        delete[] mem;
    }
} // namespace writeOutFuncs

namespace
{
    struct Task {
        float *mem;
        unsigned W, H;
        WriteOutCallBack cb;
        std::string name;
        imr_params p;
    };

    struct Queue {
        std::mutex mu;
        std::condition_variable cv;        // worker: new tasks / shutdown
        std::condition_variable cv_done;   // completer: finished tasks
        std::deque<Task> incoming;
        std::deque<std::pair<Task, int>> finished;
        std::map<long long, Task> inflight;
        bool stop = false;
        bool worker_done = false;
        long long next_tag = 1;
        int device = 0;
        std::thread worker, completer;
        bool running = false;
    };

    Queue g_q;

    void worker_loop()
    {
        cudaSetDevice(g_q.device);
        imr_engine *eng = nullptr;
        if (imr_engine_create(&eng, 0, 4096, nullptr) != IMR_SUCCESS) {
            fprintf(stderr, "imresh_b200 task queue: engine creation failed: %s\n", imr_last_error());
        }
        std::vector<imr_result> res(256);
        for (;;) {
            std::deque<std::pair<long long, Task>> fresh;
            bool stop;
            {
                std::unique_lock<std::mutex> lk(g_q.mu);
                g_q.cv.wait(lk, [&] { return g_q.stop || !g_q.incoming.empty() || !g_q.inflight.empty(); });
                while (!g_q.incoming.empty()) {
                    long long tag = g_q.next_tag++;
                    fresh.emplace_back(tag, g_q.incoming.front());
                    g_q.inflight.emplace(tag, g_q.incoming.front());
                    g_q.incoming.pop_front();
                }
                stop = g_q.stop && g_q.inflight.empty();
            }
            if (stop) break;
            for (auto &f : fresh) {
                int rc = eng ? imr_engine_submit(eng, f.second.mem, f.second.mem, f.second.W, f.second.H,
                                                 &f.second.p, f.first)
                             : IMR_ERR_NOT_INITIALIZED;
                if (rc != IMR_SUCCESS) {   // rejected: report through the callback path
                    std::lock_guard<std::mutex> lk(g_q.mu);
                    g_q.finished.emplace_back(g_q.inflight[f.first], rc);
                    g_q.inflight.erase(f.first);
                    g_q.cv_done.notify_one();
                }
            }
            if (!eng) continue;
            imr_engine_step(eng);
            int n = 0;
            imr_engine_poll(eng, res.data(), (int)res.size(), &n);
            if (n) {
                std::lock_guard<std::mutex> lk(g_q.mu);
                for (int i = 0; i < n; ++i) {
                    auto it = g_q.inflight.find(res[i].tag);
                    if (it == g_q.inflight.end()) continue;
                    g_q.finished.emplace_back(it->second, res[i].status);
                    g_q.inflight.erase(it);
                }
                g_q.cv_done.notify_one();
            }
        }
        if (eng) imr_engine_destroy(eng);
        std::lock_guard<std::mutex> lk(g_q.mu);
        g_q.worker_done = true;
        g_q.cv_done.notify_one();
    }

    void completer_loop()
    {
        for (;;) {
            std::pair<Task, int> t;
            {
                std::unique_lock<std::mutex> lk(g_q.mu);
                g_q.cv_done.wait(lk, [&] { return !g_q.finished.empty() || g_q.worker_done; });
                if (g_q.finished.empty()) return;   // worker done and nothing left
                t = g_q.finished.front();
                g_q.finished.pop_front();
            }
            if (t.second != IMR_SUCCESS)
                fprintf(stderr, "imresh_b200 task queue: task %s failed: %s\n", t.first.name.c_str(),
                        imr_status_string(t.second));
            if (t.first.cb) t.first.cb(t.first.mem, t.first.W, t.first.H, t.first.name);
        }
    }
} // namespace

void taskQueueInit()
{
    std::lock_guard<std::mutex> lk(g_q.mu);
    if (g_q.running) return;
    cudaGetDevice(&g_q.device);
    g_q.stop = false;
    g_q.worker_done = false;
    g_q.worker = std::thread(worker_loop);
    g_q.completer = std::thread(completer_loop);
    g_q.running = true;
}

void addTask(float *const ioData, unsigned int const imageWidth, unsigned int const imageHeight,
             WriteOutCallBack writeOutFunc, std::string fileName, unsigned int nCycles, unsigned int nHioCycles,
             float targetError, float hioBeta, float intensityCutOffAutoCorel, float intensityCutOff,
             float sigma0, float sigmaChange)
{
    // the reference forwards these to cudaShrinkWrap (taskQueue.cu:129-142),
    // whose <= 0 defaults apply
    Task t{ioData, imageWidth, imageHeight, std::move(writeOutFunc), std::move(fileName),
           imr_params{nCycles, targetError, hioBeta, intensityCutOffAutoCorel, intensityCutOff, sigma0,
                      sigmaChange, nHioCycles}};
    std::lock_guard<std::mutex> lk(g_q.mu);
    if (!g_q.running) {
        fprintf(stderr, "imresh_b200 task queue: addTask before taskQueueInit\n");
        return;
    }
    g_q.incoming.push_back(std::move(t));
    g_q.cv.notify_one();
}

void taskQueueDeinit()
{
    {
        std::lock_guard<std::mutex> lk(g_q.mu);
        if (!g_q.running) return;
        g_q.stop = true;
        g_q.cv.notify_one();
    }
    g_q.worker.join();
    g_q.completer.join();
    std::lock_guard<std::mutex> lk(g_q.mu);
    g_q.running = false;
}

} // namespace io
} // namespace imresh
