/* ORACLE / TEST INFRASTRUCTURE -- not part of the product.
 *
 * Forced include (g++ -include) for compiling the reference's
 * examples/threadedExample.cpp unmodified.  Without USE_SPLASH that file
 * names ImageDimensions without its namespace (threadedExample.cpp:52, in
 * the reference's tree), which the reference's own headers declare only as
 * imresh::io::readInFuncs::ImageDimensions
 * (src/imresh/io/readInFuncs/readInFuncs.hpp:40), so it does not compile
 * against the reference either; this using-declaration supplies the name. */
#pragma once
#include "io/readInFuncs/readInFuncs.hpp"
using imresh::io::readInFuncs::ImageDimensions;
