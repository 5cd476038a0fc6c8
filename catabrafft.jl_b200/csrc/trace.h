// trace.h -- NVTX ranges around the library's host entry points (plan
// creation, execution, the host-buffer pipeline, the batched and serving
// forms, wisdom files), in the NVTX domain "catabra_b200".  NVTX3 is
// header-only: with no tool attached a range costs a load and a branch, and
// a profiler (or any NVTX injection library named by NVTX_INJECTION64_PATH)
// sees every call as a named range on the calling thread.
#pragma once
#include <nvtx3/nvToolsExt.h>

#include <cstdarg>
#include <cstdio>

namespace cfft_trace {

inline nvtxDomainHandle_t domain() {
    static nvtxDomainHandle_t d = nvtxDomainCreateA("catabra_b200");
    return d;
}

// one range for the lifetime of the object; the message is copied at push
class Range {
public:
    explicit Range(const char* msg) { push(msg); }
    Range(const char* fmt, long long a, long long b, long long c = 0, long long d = 0) {
        char buf[160];
        snprintf(buf, sizeof buf, fmt, a, b, c, d);
        push(buf);
    }
    ~Range() { nvtxDomainRangePop(domain()); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;

private:
    static void push(const char* msg) {
        nvtxEventAttributes_t a = {};
        a.version = NVTX_VERSION;
        a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
        a.messageType = NVTX_MESSAGE_TYPE_ASCII;
        a.message.ascii = msg;
        nvtxDomainRangePushEx(domain(), &a);
    }
};

}  // namespace cfft_trace
