/*
 * Read-in functions for task inputs, with the reference's types
 * (src/imresh/io/readInFuncs/readInFuncs.hpp:57-84): a FloatImage is the
 * image buffer and (width, height).  The buffer comes from new[]; ownership
 * passes to the caller (addTask hands it on to the write-out callback, which
 * releases it).  Formats that need no third-party library:
 *   readTxt   whitespace-separated numbers, one image row per line (the
 *             reference's readTxt returns a pointer to a stack array that is
 *             gone on return, readInFuncs.cpp:84-91; this one does not)
 *   readNpy   NumPy .npy, float32 or float64, 1-D or 2-D, C order
 * On failure the buffer is NULL and (0, 0) is returned, with a message on
 * stderr (the reference exits the process).
 */
#pragma once
#include <string>
#include <utility>

namespace imresh
{
namespace io
{
namespace readInFuncs
{
    using ImageDimensions = std::pair< unsigned int, unsigned int >;
    using FloatImage = std::pair< float *, ImageDimensions >;

    FloatImage readTxt( std::string const filename );
    FloatImage readNpy( std::string const filename );
} // namespace readInFuncs
} // namespace io
} // namespace imresh
