/*
 * The write-out callback of the reference that needs no file-format
 * library: justFree (src/imresh/io/writeOutFuncs/writeOutFuncs.hpp:52-57)
 * releases the task's buffer with delete[] and ignores the other arguments.
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
} // namespace writeOutFuncs
} // namespace io
} // namespace imresh
