/* Stand-in for the one TBB type the reference's host queue uses
 * (src/pipe.h:4,17: tbb::mutex with lock()/unlock()).  TBB is not installed
 * here; std::mutex has the same interface.  Used only to compile the
 * reference sources into oracle/_ref (test infrastructure). */
#pragma once
#include <mutex>
namespace tbb { using mutex = std::mutex; }
