// mdl_runtime.cuh — the argument-block and read-only-data readers of the MDL
// runtime (shaders/mdl_runtime.hlsl:24-75), the entry points through which
// MDL SDK-generated material code reads its parameters.  The buffers are
// HLSL ByteAddressBuffers: Load(offs) returns the 32-bit word at offs with
// its two low bits ignored.  A read past the end returns 0 (the robust
// buffer access of the reference's Vulkan device); these readers never fault.
#pragma once
#include <cstdint>

namespace sb {

__device__ __forceinline__ uint32_t mdl_load_word(const uint8_t* base, uint64_t bytes, uint32_t offs)
{
    const uint64_t a = (uint64_t)(offs & ~3u);
    if (!base || a + 4 > bytes) return 0u;
    return __ldg(reinterpret_cast<const uint32_t*>(base + a));
}

__device__ __forceinline__ float mdl_read_as_float(const uint8_t* base, uint64_t bytes, uint32_t offs)
{
    return __uint_as_float(mdl_load_word(base, bytes, offs));
}

// asdouble(Load(offs), Load(offs + 4)): low word first
__device__ __forceinline__ double mdl_read_as_double(const uint8_t* base, uint64_t bytes, uint32_t offs)
{
    const uint64_t lo = mdl_load_word(base, bytes, offs), hi = mdl_load_word(base, bytes, offs + 4u);
    return __longlong_as_double((long long)((hi << 32) | lo));
}

__device__ __forceinline__ int32_t mdl_read_as_int(const uint8_t* base, uint64_t bytes, uint32_t offs)
{
    return (int32_t)mdl_load_word(base, bytes, offs);
}

__device__ __forceinline__ uint32_t mdl_read_as_uint(const uint8_t* base, uint64_t bytes, uint32_t offs)
{
    return mdl_load_word(base, bytes, offs);
}

// the byte at offs of its aligned word is nonzero
__device__ __forceinline__ bool mdl_read_as_bool(const uint8_t* base, uint64_t bytes, uint32_t offs)
{
    const uint32_t val = mdl_load_word(base, bytes, offs & ~3u);
    return (val & (0xffu << (8u * (offs & 3u)))) != 0u;
}

}  // namespace sb
