// common.cpp — error reporting, version and layout queries of the C ABI.
#include "common.h"

#include <cstdlib>
#include <cstring>

namespace sb {
std::string& last_error()
{
    thread_local std::string msg;
    return msg;
}
}  // namespace sb

extern "C" int strelka_get_last_error(char* buffer, size_t capacity)
{
    const std::string& m = sb::last_error();
    if (buffer && capacity) {
        size_t n = m.size() < capacity - 1 ? m.size() : capacity - 1;
        memcpy(buffer, m.data(), n);
        buffer[n] = '\0';
    }
    return (int)m.size();
}

extern "C" int strelka_version(void) { return 100; }

extern "C" size_t strelka_sizeof(const char* name)
{
    if (!name) return 0;
#define SB_SZ(T) \
    if (strcmp(name, #T) == 0) return sizeof(T);
    SB_SZ(PathTracerParam)
    SB_SZ(AccumulationParam)
    SB_SZ(Tonemapparam)
    SB_SZ(BVHNode)
    SB_SZ(Vertex)
    SB_SZ(InstanceConstants)
    SB_SZ(UniformLight)
    SB_SZ(MdlMaterial)
    SB_SZ(Mdl_resource_info)
    SB_SZ(Ray)
    SB_SZ(Hit)
    SB_SZ(BVHInputPosition)
    SB_SZ(StrelkaMaterialArgs)
    SB_SZ(StrelkaTexture)
    SB_SZ(StrelkaEnvMap)
    SB_SZ(PathTracerDesc)
    SB_SZ(ReductionDesc)
    SB_SZ(AccumulationDesc)
    SB_SZ(TonemapDesc)
    SB_SZ(Upscalepassparam)
    SB_SZ(UpscaleDesc)
    SB_SZ(StrelkaUsdLight)
    SB_SZ(TraceDesc)
    SB_SZ(StrelkaPathTracerConfig)
    SB_SZ(StrelkaNrcRecord)
    SB_SZ(StrelkaNrcConfig)
    SB_SZ(StrelkaNrcRenderConfig)
    SB_SZ(StrelkaBatchConfig)
    SB_SZ(StrelkaBatchTuneEntry)
#undef SB_SZ
    return 0;
}

extern "C" void strelka_host_free(void* p) { free(p); }
