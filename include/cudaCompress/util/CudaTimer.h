// util/CudaTimer.h - named event timers (reference util/CudaTimer.h:19-72).
// Kept for source compatibility; timing of this library is done with CUDA
// events by its own benchmark, so these record nothing.
#ifndef CUDACOMPRESS_B200_CUDA_TIMER_H
#define CUDACOMPRESS_B200_CUDA_TIMER_H

#include <map>
#include <string>
#include <vector>

#include <cudaCompress/global.h>

namespace cudaCompress {
namespace util {

class CudaTimerResources {
public:
    CudaTimerResources(bool enabled = false) : m_isEnabled(enabled) {}
    void setEnabled(bool enable = true) { m_isEnabled = enable; }
    const std::map<std::string, float>& getAccumulatedTimes(bool) { return m_times; }
    void getAccumulatedTimes(std::vector<std::string>& names, std::vector<float>& times, bool) {
        for (const auto& kv : m_times) { names.push_back(kv.first); times.push_back(kv.second); }
    }
    void reset() { m_times.clear(); }
    void record(const std::string&) {}

private:
    bool m_isEnabled;
    std::map<std::string, float> m_times;
};

class CudaScopedTimer {
public:
    CudaScopedTimer(CudaTimerResources& resources) : m_resources(resources) {}
    void operator()(const std::string& = std::string()) {}

private:
    CudaTimerResources& m_resources;
};

}
}

#endif
