// Host helpers the reference's applications use from src/tools.h: wtime(),
// wall-clock seconds (app/bfs.cu:146-160 times App::run with it).
#ifndef SCAPH_COMPAT_TOOLS_H
#define SCAPH_COMPAT_TOOLS_H

#include <sys/time.h>

inline double wtime()
{
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (double)tv.tv_sec + (double)tv.tv_usec * 1e-6;
}

#endif
