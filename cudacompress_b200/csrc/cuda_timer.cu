// cuda_timer.cu - util::CudaTimerResources / CudaScopedTimer (host code;
// reference util/CudaTimer.cpp semantics): a section runs from the event of
// its record(name) to the next recorded event; unnamed records only end a
// section.  Events are reused once accounted.
#include <cudaCompress/util/CudaTimer.h>

namespace cudaCompress {
namespace util {

CudaTimerResources::CudaTimerResources(bool enabled) : m_isEnabled(enabled) {}

CudaTimerResources::~CudaTimerResources() {
    reset();
    for (cudaEvent_t e : m_free) cudaEventDestroy(e);
}

cudaEvent_t CudaTimerResources::takeEvent() {
    if (m_free.empty()) account(false);
    if (m_free.empty()) {
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    cudaEvent_t e = m_free.back();
    m_free.pop_back();
    return e;
}

void CudaTimerResources::record(const std::string& name) {
    if (!m_isEnabled) return;
    Mark m;
    m.name = name;
    m.event = takeEvent();
    cudaEventRecord(m.event);
    m_pending.push_back(m);
}

void CudaTimerResources::account(bool sync) {
    while (!m_pending.empty()) {
        Mark& next = m_pending.front();
        if (m_open.event) {
            if (sync) cudaEventSynchronize(next.event);
            else if (cudaEventQuery(next.event) != cudaSuccess) return;   // not reached on the GPU yet
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, m_open.event, next.event);
            m_times[m_open.name] += ms;
            m_free.push_back(m_open.event);
            m_open = Mark();
        }
        if (next.name.empty()) m_free.push_back(next.event);
        else m_open = next;
        m_pending.pop_front();
    }
}

const std::map<std::string, float>& CudaTimerResources::getAccumulatedTimes(bool sync) {
    account(sync);
    return m_times;
}

void CudaTimerResources::getAccumulatedTimes(std::vector<std::string>& names, std::vector<float>& times, bool sync) {
    for (const auto& kv : getAccumulatedTimes(sync)) {
        names.push_back(kv.first);
        times.push_back(kv.second);
    }
}

void CudaTimerResources::reset() {
    if (m_open.event) m_free.push_back(m_open.event);
    m_open = Mark();
    for (const Mark& m : m_pending) m_free.push_back(m.event);
    m_pending.clear();
    m_times.clear();
}

CudaScopedTimer::CudaScopedTimer(CudaTimerResources& resources) : m_resources(resources), m_sectionOpen(false) {}

CudaScopedTimer::~CudaScopedTimer() {
    if (m_sectionOpen) m_resources.record(std::string());
}

void CudaScopedTimer::operator()(const std::string& name) {
    if (name.empty() && !m_sectionOpen) return;
    m_resources.record(name);
    m_sectionOpen = !name.empty();
}

}  // namespace util
}  // namespace cudaCompress
