// Shared host/device vector math and data layouts of the B200 path-tracing core.
//
// Conventions that the rest of the core relies on:
//   * geometry, BSDF and MIS arithmetic is FP32; the film accumulators are FP64;
//   * functions whose results must match the reference bit for bit (the watertight triangle
//     test, Engine/Source/Math/Geometry/TWatertightTriangle.ipp:16-149) use the explicitly
//     rounded intrinsics (__fmul_rn / __fadd_rn / __fsub_rn / __fdiv_rn) so that nvcc cannot
//     contract them into FMAs; everything else may contract freely.
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define PG_HD __host__ __device__ __forceinline__
#else
#define PG_HD inline
#endif

namespace pg
{

#if !defined(__CUDACC__)
using std::isfinite;
using std::sqrt;
inline float fmaxf(float a, float b) { return std::fmax(a, b); }
inline float fminf(float a, float b) { return std::fmin(a, b); }
#endif

struct V3
{
	float x, y, z;
};

PG_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
PG_HD V3 operator + (V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
PG_HD V3 operator - (V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
PG_HD V3 operator - (V3 a) { return V3{-a.x, -a.y, -a.z}; }
PG_HD V3 operator * (V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
PG_HD V3 operator * (float s, V3 a) { return V3{a.x * s, a.y * s, a.z * s}; }
PG_HD V3 operator * (V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
PG_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PG_HD V3 cross(V3 a, V3 b)
{
	return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
PG_HD float length_sq(V3 a) { return dot(a, a); }
PG_HD float length(V3 a) { return std::sqrt(dot(a, a)); }
PG_HD V3 normalize(V3 a)
{
	const float rcp = 1.0f / std::sqrt(dot(a, a));
	return a * rcp;
}
PG_HD bool is_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
PG_HD bool is_finite(V3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
PG_HD float max3(float a, float b, float c) { return fmaxf(a, fmaxf(b, c)); }
PG_HD float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// Finite values are clamped, non-finite ones map to the lower bound
// (Engine/Source/Math/math.h:98-111, `safe_clamp`).
PG_HD float safe_clamp(float v, float lo, float hi)
{
	return isfinite(v) ? clampf(v, lo, hi) : lo;
}

// ---------------------------------------------------------------------------------------------
// Compressed 8-wide BVH node (80 bytes = 5 x 16-byte words), child boxes quantized to 8 bits per
// plane relative to the node origin `p` with a power-of-two scale per axis.
//
//   w0: p.x, p.y, p.z (float), [e.x | e.y << 8 | e.z << 16 | imask << 24]
//   w1: child_base, tri_base, meta[0..3], meta[4..7]
//   w2: qlo.x[0..7] (2 words), qlo.y[0..7] (2 words)
//   w3: qlo.z[0..7], qhi.x[0..7]
//   w4: qhi.y[0..7], qhi.z[0..7]
//
// meta byte of slot s: 0 = empty; internal child: 0b001 << 5 | (24 + s); leaf child with n
// triangles (1..3): unary(n) << 5 | offset, where offset is the first triangle relative to
// tri_base. imask bit s marks an internal child; internal children are stored contiguously
// from child_base in slot order. Slot s of a child is chosen so that the bits of s encode the
// octant its centroid lies in relative to the parent (bit set = negative side), which lets the
// traversal visit children front to back with one XOR per ray octant.
struct alignas(16) WideNode
{
	uint32_t w[20];
};
static_assert(sizeof(WideNode) == 80, "wide node must be 80 bytes");

// One triangle as stored for traversal and shading, in BVH leaf order: 3 x float4.
//   v0.xyz, w = original primitive index (bit pattern of a uint32)
//   v1.xyz, w = material index
//   v2.xyz, w = emitter index + 1 (0 = not an emitter)
struct alignas(16) LeafTri
{
	float v0x, v0y, v0z; uint32_t prim;
	float v1x, v1y, v1z; uint32_t material;
	float v2x, v2y, v2z; uint32_t emitter_plus_one;
};
static_assert(sizeof(LeafTri) == 48, "leaf triangle must be 48 bytes");

// Error codes reported through the C ABI (0 = success).
enum Status : int
{
	PG_OK = 0,
	PG_ERR_INVALID_ARGUMENT = 1,
	PG_ERR_CUDA = 2,
	PG_ERR_NOT_FOUND = 3,
	PG_ERR_STACK_OVERFLOW = 4,
	PG_ERR_QUEUE_OVERFLOW = 5,
	PG_ERR_SCENE = 6,
	PG_ERR_NO_DEVICE = 7,
	PG_ERR_ITERATION_LIMIT = 8,
};

// Device-side error flags written by kernels (bitwise OR into one word).
enum DeviceErrorFlag : uint32_t
{
	PG_DEV_ERR_STACK = 1u << 0,
	PG_DEV_ERR_QUEUE = 1u << 1,
	PG_DEV_ERR_NAN = 1u << 2,
	PG_DEV_ERR_GUIDE_WAIT = 1u << 3,   // a guiding-network kernel gave up waiting on its tensor cores
};

// Traversal stack depth (node groups). The builder checks the tree depth against it.
constexpr int kTraversalStackSize = 64;

}// end namespace pg
