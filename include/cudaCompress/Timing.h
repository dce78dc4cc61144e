// Timing.h - timing queries (reference Timing.h:15-27).  This library times
// its kernels with CUDA events in its own tools; these calls are accepted and
// report no sections.
#ifndef CUDACOMPRESS_B200_TIMING_H
#define CUDACOMPRESS_B200_TIMING_H

#include <string>
#include <vector>

#include <cudaCompress/global.h>

namespace cudaCompress {

class Instance;

enum ETimingDetail {
    TIMING_DETAIL_NONE,
    TIMING_DETAIL_LOW,
    TIMING_DETAIL_MEDIUM,
    TIMING_DETAIL_HIGH,
};

void CUCOMP_DLL setTimingDetail(Instance* pCudaCompressInstance, ETimingDetail detail);
void CUCOMP_DLL getTimings(Instance* pCudaCompressInstance, std::vector<std::string>& names, std::vector<float>& times);
void CUCOMP_DLL printTimings(Instance* pCudaCompressInstance);
void CUCOMP_DLL resetTimings(Instance* pCudaCompressInstance);

}

#endif
