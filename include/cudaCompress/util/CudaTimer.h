// util/CudaTimer.h - named sections timed with CUDA events (drop-in for the
// reference's include/cudaCompress/util/CudaTimer.h:19-72).  record(name)
// marks the end of the running section and, for a non-empty name, the start
// of section `name`; elapsed times add up per name.  Events are recorded on
// the default stream, as the reference does.
#ifndef CUDACOMPRESS_B200_CUDA_TIMER_H
#define CUDACOMPRESS_B200_CUDA_TIMER_H

#include <deque>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include <cudaCompress/global.h>

namespace cudaCompress {
namespace util {

class CudaTimerResources {
public:
    CUCOMP_DLL CudaTimerResources(bool enabled = false);
    CUCOMP_DLL ~CudaTimerResources();

    void setEnabled(bool enable = true) { m_isEnabled = enable; }

    // accumulated milliseconds per section name; sync waits for every
    // recorded event, otherwise only finished ones are accounted
    CUCOMP_DLL const std::map<std::string, float>& getAccumulatedTimes(bool sync);
    CUCOMP_DLL void getAccumulatedTimes(std::vector<std::string>& names, std::vector<float>& times, bool sync);
    CUCOMP_DLL void reset();

    CUCOMP_DLL void record(const std::string& name);

private:
    struct Mark {
        std::string name;
        cudaEvent_t event = nullptr;
    };
    void account(bool sync);
    cudaEvent_t takeEvent();

    bool m_isEnabled;
    std::deque<Mark> m_pending;      // recorded, not yet accounted
    Mark m_open;                     // start of the section being timed
    std::vector<cudaEvent_t> m_free;
    std::map<std::string, float> m_times;
};

// Times consecutive sections of a scope: timer("a"); ... timer("b"); ...
// timer() (or the end of the scope) closes the last one.
class CudaScopedTimer {
public:
    CUCOMP_DLL CudaScopedTimer(CudaTimerResources& resources);
    CUCOMP_DLL ~CudaScopedTimer();

    CUCOMP_DLL void operator()(const std::string& name = std::string());

private:
    CudaTimerResources& m_resources;
    bool m_sectionOpen;
};

}
}

#endif
