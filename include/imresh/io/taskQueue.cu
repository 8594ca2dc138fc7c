/*
 * The reference's examples include "io/taskQueue.cu" directly
 * (examples/threadedExample.cpp:32, examples/outputExampleCreation.cpp:30).
 * This file keeps that include line working: the implementation lives in
 * libimresh_b200.so, so it only pulls in the declarations.
 */
#pragma once
#include "taskQueue.hpp"
