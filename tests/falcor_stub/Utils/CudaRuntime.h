// Stand-in for Falcor's Utils/CudaRuntime.h: the CUDA runtime API without
// its global vector types (float3, uint2, ...), which would clash with
// Falcor's own under `using namespace Falcor`.  Each is included under a
// cuda_ prefix.  TEST INFRASTRUCTURE ONLY.
#pragma once

#define char1 cuda_char1
#define char2 cuda_char2
#define char3 cuda_char3
#define char4 cuda_char4
#define uchar1 cuda_uchar1
#define uchar2 cuda_uchar2
#define uchar3 cuda_uchar3
#define uchar4 cuda_uchar4
#define short1 cuda_short1
#define short2 cuda_short2
#define short3 cuda_short3
#define short4 cuda_short4
#define ushort1 cuda_ushort1
#define ushort2 cuda_ushort2
#define ushort3 cuda_ushort3
#define ushort4 cuda_ushort4
#define int1 cuda_int1
#define int2 cuda_int2
#define int3 cuda_int3
#define int4 cuda_int4
#define uint1 cuda_uint1
#define uint2 cuda_uint2
#define uint3 cuda_uint3
#define uint4 cuda_uint4
#define long1 cuda_long1
#define long2 cuda_long2
#define long3 cuda_long3
#define long4 cuda_long4
#define ulong1 cuda_ulong1
#define ulong2 cuda_ulong2
#define ulong3 cuda_ulong3
#define ulong4 cuda_ulong4
#define longlong1 cuda_longlong1
#define longlong2 cuda_longlong2
#define longlong3 cuda_longlong3
#define longlong4 cuda_longlong4
#define ulonglong1 cuda_ulonglong1
#define ulonglong2 cuda_ulonglong2
#define ulonglong3 cuda_ulonglong3
#define ulonglong4 cuda_ulonglong4
#define float1 cuda_float1
#define float2 cuda_float2
#define float3 cuda_float3
#define float4 cuda_float4
#define double1 cuda_double1
#define double2 cuda_double2
#define double3 cuda_double3
#define double4 cuda_double4
#include <cuda_runtime.h>
#undef char1
#undef char2
#undef char3
#undef char4
#undef uchar1
#undef uchar2
#undef uchar3
#undef uchar4
#undef short1
#undef short2
#undef short3
#undef short4
#undef ushort1
#undef ushort2
#undef ushort3
#undef ushort4
#undef int1
#undef int2
#undef int3
#undef int4
#undef uint1
#undef uint2
#undef uint3
#undef uint4
#undef long1
#undef long2
#undef long3
#undef long4
#undef ulong1
#undef ulong2
#undef ulong3
#undef ulong4
#undef longlong1
#undef longlong2
#undef longlong3
#undef longlong4
#undef ulonglong1
#undef ulonglong2
#undef ulonglong3
#undef ulonglong4
#undef float1
#undef float2
#undef float3
#undef float4
#undef double1
#undef double2
#undef double3
#undef double4
