/*
 * Write-out callbacks of the task queue (the WriteOutCallBack signature of
 * src/imresh/io/taskQueue.hpp:38-44), as the reference's
 * src/imresh/io/writeOutFuncs/writeOutFuncs.hpp:52-106 declares them, for
 * formats that need no third-party library:
 *   justFree                      releases the buffer with delete[] (hpp:52-57)
 *   writeOutNpy / AndFreeNpy      NumPy .npy, float32, shape (height, width)
 *   writeOutTxt / AndFreeTxt      text, one image row per line
 *   writeOutRaw / AndFreeRaw      headerless float32, width contiguous
 * The *AndFree forms release the buffer with delete[] after writing, as the
 * reference's writeOutAndFreePNG / HDF5 do (the PNG and HDF5 writers need
 * pngwriter and libSplash, which are not part of this build).  A write that
 * fails prints to stderr (the reference exits the process).
 */
#pragma once
#include <string>

namespace imresh
{
namespace io
{
namespace writeOutFuncs
{
    void justFree(
        float * mem,
        unsigned int const imageWidth,
        unsigned int const imageHeight,
        std::string const fileName
    );
    void writeOutNpy( float * mem, unsigned int const imageWidth, unsigned int const imageHeight,
                      std::string const fileName );
    void writeOutAndFreeNpy( float * mem, unsigned int const imageWidth, unsigned int const imageHeight,
                             std::string const fileName );
    void writeOutTxt( float * mem, unsigned int const imageWidth, unsigned int const imageHeight,
                      std::string const fileName );
    void writeOutAndFreeTxt( float * mem, unsigned int const imageWidth, unsigned int const imageHeight,
                             std::string const fileName );
    void writeOutRaw( float * mem, unsigned int const imageWidth, unsigned int const imageHeight,
                      std::string const fileName );
    void writeOutAndFreeRaw( float * mem, unsigned int const imageWidth, unsigned int const imageHeight,
                             std::string const fileName );
} // namespace writeOutFuncs
} // namespace io
} // namespace imresh
