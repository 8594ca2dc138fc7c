/*
 * Drop-in declarations of the reference's batch front end
 * (src/imresh/io/taskQueue.hpp:38-84), implemented by libimresh_b200.so.
 *
 * Behaviour kept from the reference: addTask takes ownership of ioData (the
 * Fourier modulus, overwritten with the reconstruction) and hands it to
 * writeOutFunc(ioData, width, height, fileName) when the task is done; the
 * callback runs on a library thread, concurrently with the caller, and owns
 * freeing the buffer; addTask must be called between taskQueueInit and
 * taskQueueDeinit from one producer thread; taskQueueDeinit waits for every
 * task and callback.
 *
 * Behaviour that differs by design: tasks are not run one std::thread per
 * task on rotating streams; they are queued to one device-resident batched
 * engine (imr_engine_*) on the current CUDA device that advances all admitted
 * reconstructions together, so addTask never blocks on a full pool.
 */
#pragma once

#include <functional>
#include <string>

namespace imresh
{
namespace io
{
    using WriteOutCallBack = std::function<
                                 void ( float *,
                                        unsigned int const,
                                        unsigned int const,
                                        std::string )
                             >;

    void addTask(
        float * const ioData,
        unsigned int const imageWidth                   ,
        unsigned int const imageHeight                  ,
        WriteOutCallBack writeOutFunc                   ,
        std::string      fileName                       ,
        unsigned int     nCycles                  = 20  ,
        unsigned int     nHioCycles               = 20  ,
        float            targetError              = 1e-5,
        float            hioBeta                  = 0.9f,
        float            intensityCutOffAutoCorel = 0.04,
        float            intensityCutOff          = 0.2 ,
        float            sigma0                   = 3.0 ,
        float            sigmaChange              = 0.01
    );

    /* First call of the library: starts the engine and its threads. */
    void taskQueueInit( );

    /* Last call: waits for every task and write-out callback, then stops. */
    void taskQueueDeinit( );

} // namespace io
} // namespace imresh
