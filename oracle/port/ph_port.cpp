// CPU restatement of the reference BNEEPT / BVPT path (test infrastructure only: the oracle and,
// where the reference build is unavailable, the CPU baseline). Plain scalar C++17, no FMA
// contraction (built with -ffp-contract=off), every function citing the reference code it
// restates (paths relative to Engine/Engine/Source/ of the reference).
//
// Library (C ABI, loaded by the tests through ctypes) and CLI:
//   ph_port_render <scene.bin> <threads> <max-bounces> <out.rgbf32> [repeats]
// scene.bin (little-endian): "PHPT" u32 version=1, u32 width, height, spp, estimator (0 BNEEPT,
//   1 BVPT, 2 BVPTDL), f32 camera[12] (pos, dir, up, fov, width, height), u32 num_tris, num_materials,
//   num_emitters, f32 tris[n][9], u32 tri_material[n], u32 tri_emitter[n] (index + 1),
//   f32 materials[m][8], f32 emitters[e][4] -- the layout of pgpu_scene_create.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>

namespace port
{

struct Vec
{
	float x = 0, y = 0, z = 0;
};
inline Vec mk(float x, float y, float z) { return Vec{x, y, z}; }
inline Vec operator + (Vec a, Vec b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline Vec operator - (Vec a, Vec b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline Vec operator - (Vec a) { return mk(-a.x, -a.y, -a.z); }
inline Vec operator * (Vec a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline float dot(Vec a, Vec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec cross(Vec a, Vec b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float len(Vec a) { return std::sqrt(dot(a, a)); }
// TVectorNBase::normalize -> math::normalize: multiply by 1 / length (Math/math.ipp:154-163)
inline Vec unit(Vec a) { const float r = 1.0f / len(a); return a * r; }
inline bool is_zero(Vec a) { return a.x == 0 && a.y == 0 && a.z == 0; }

struct Rgb
{
	float r = 0, g = 0, b = 0;
};
inline Rgb operator * (Rgb a, Rgb b) { return Rgb{a.r * b.r, a.g * b.g, a.b * b.b}; }
inline Rgb operator * (Rgb a, float s) { return Rgb{a.r * s, a.g * s, a.b * s}; }
inline Rgb operator + (Rgb a, Rgb b) { return Rgb{a.r + b.r, a.g + b.g, a.b + b.b}; }
inline bool finite(Rgb a) { return std::isfinite(a.r) && std::isfinite(a.g) && std::isfinite(a.b); }
inline bool zero(Rgb a) { return a.r == 0 && a.g == 0 && a.b == 0; }
// math::safe_clamp (Math/math.h:98-111)
inline float safe_clamp(float v, float lo, float hi) { return std::isfinite(v) ? std::min(std::max(v, lo), hi) : lo; }
inline Rgb safe_clamp(Rgb a) { return Rgb{safe_clamp(a.r, 0, 1e9f), safe_clamp(a.g, 0, 1e9f), safe_clamp(a.b, 0, 1e9f)}; }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kFltMax = std::numeric_limits<float>::max();

// ----------------------------------------------------------------------------------------------
// Watertight ray/triangle test: Math/Geometry/TWatertightTriangle.ipp:16-149.
bool watertight(Vec o, Vec d, float min_t, float max_t, Vec va, Vec vb, Vec vc, float* out_t, float b[3])
{
	Vec dir = d;
	Vec a = va - o, bb = vb - o, c = vc - o;
	auto perm = [](Vec v, int k) { return k == 0 ? mk(v.y, v.z, v.x) : mk(v.z, v.x, v.y); };
	if(std::abs(dir.x) > std::abs(dir.y))
	{
		if(std::abs(dir.x) > std::abs(dir.z)) { dir = perm(dir, 0); a = perm(a, 0); bb = perm(bb, 0); c = perm(c, 0); }
	}
	else if(std::abs(dir.y) > std::abs(dir.z))
	{
		dir = perm(dir, 1); a = perm(a, 1); bb = perm(bb, 1); c = perm(c, 1);
	}
	const float rz = 1.0f / dir.z;
	const float sx = -dir.x * rz, sy = -dir.y * rz, sz = rz;
	a.x += sx * a.z; a.y += sy * a.z;
	bb.x += sx * bb.z; bb.y += sy * bb.z;
	c.x += sx * c.z; c.y += sy * c.z;
	float ea = bb.x * c.y - bb.y * c.x;
	float eb = c.x * a.y - c.y * a.x;
	float ec = a.x * bb.y - a.y * bb.x;
	if(ea == 0 || eb == 0 || ec == 0)
	{
		ea = static_cast<float>(static_cast<double>(bb.x) * c.y - static_cast<double>(bb.y) * c.x);
		eb = static_cast<float>(static_cast<double>(c.x) * a.y - static_cast<double>(c.y) * a.x);
		ec = static_cast<float>(static_cast<double>(a.x) * bb.y - static_cast<double>(a.y) * bb.x);
	}
	if((ea < 0 || eb < 0 || ec < 0) && (ea > 0 || eb > 0 || ec > 0))
	{
		return false;
	}
	const float det = ea + eb + ec;
	if(det == 0 || !std::isfinite(det))
	{
		return false;
	}
	a.z *= sz; bb.z *= sz; c.z *= sz;
	const float ts = ea * a.z + eb * bb.z + ec * c.z;
	if(det > 0) { if(ts < min_t * det || ts > max_t * det) { return false; } }
	else        { if(ts > min_t * det || ts < max_t * det) { return false; } }
	const float rd = 1.0f / det;
	b[0] = ea * rd; b[1] = eb * rd; b[2] = ec * rd;
	*out_t = ts * rd;
	return true;
}

// ----------------------------------------------------------------------------------------------
// Scene with a plain binary BVH (median split). The closest hit does not depend on the tree:
// every triangle is bounded conservatively and ties are resolved to the smaller index.

struct Tri
{
	Vec a, b, c;
	uint32_t material, emitter;   // emitter index + 1
};

struct Material
{
	int type;          // 0 matte, 1 conductor, 2 dielectric
	Rgb c;             // albedo or F0
	float alpha;
	float ior_outer, ior_inner;
};

struct Emitter
{
	Rgb radiance;
	int type;                      // 0 triangles, 1 constant environment
	std::vector<uint32_t> tris;
	double weight = 0;
	float pmf = 0;
};

struct Node
{
	float lo[3], hi[3];
	int left = -1, right = -1;
	uint32_t begin = 0, count = 0;
};

struct Scene
{
	uint32_t width = 0, height = 0, spp = 1, estimator = 0;
	std::vector<Tri> tris;
	std::vector<Material> materials;
	std::vector<Emitter> emitters;
	std::vector<float> cdf;        // emitter pick CDF (TPwcDistribution1D semantics)
	int env = -1;
	Rgb env_radiance;
	// the dome (LatLongEnvEmitter over PLatLongEnvSphere): lat-long image (row 0 = bottom; a
	// constant environment is 1 x 1), rotation, sphere, and the texel distribution
	// (TPwcDistribution2D: marginal CDF over rows, conditional CDFs within rows)
	uint32_t env_w = 0, env_h = 0;
	std::vector<Rgb> env_texels;
	double env_rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
	double env_center[3] = {0, 0, 0};
	double env_radius = 1;
	bool env_exact = false;
	std::vector<double> env_row_cdf;    // [h + 1]
	std::vector<double> env_col_cdf;    // [h][w + 1]
	std::vector<double> env_pdf_uv;     // [h][w]
	// camera
	Vec cam_pos, ax, ay, az;
	float sensor_w = 0, sensor_h = 0, sensor_offset = 0;
	// BVH
	std::vector<Node> nodes;
	std::vector<uint32_t> order;
};

void build_bvh(Scene& s)
{
	const uint32_t n = static_cast<uint32_t>(s.tris.size());
	s.order.resize(n);
	for(uint32_t i = 0; i < n; ++i) { s.order[i] = i; }
	std::vector<float> cen(3 * n);
	for(uint32_t i = 0; i < n; ++i)
	{
		const Tri& t = s.tris[i];
		cen[3 * i + 0] = (t.a.x + t.b.x + t.c.x) / 3;
		cen[3 * i + 1] = (t.a.y + t.b.y + t.c.y) / 3;
		cen[3 * i + 2] = (t.a.z + t.b.z + t.c.z) / 3;
	}
	s.nodes.clear();
	s.nodes.reserve(2 * n);
	struct Job { int node; uint32_t b, e; };
	std::vector<Job> stack;
	s.nodes.push_back(Node{});
	stack.push_back({0, 0, n});
	while(!stack.empty())
	{
		const Job j = stack.back();
		stack.pop_back();
		Node& nd = s.nodes[j.node];
		for(int a = 0; a < 3; ++a) { nd.lo[a] = kFltMax; nd.hi[a] = -kFltMax; }
		for(uint32_t i = j.b; i < j.e; ++i)
		{
			const Tri& t = s.tris[s.order[i]];
			for(const Vec& v : {t.a, t.b, t.c})
			{
				const float c[3] = {v.x, v.y, v.z};
				for(int a = 0; a < 3; ++a) { nd.lo[a] = std::min(nd.lo[a], c[a]); nd.hi[a] = std::max(nd.hi[a], c[a]); }
			}
		}
		for(int a = 0; a < 3; ++a)
		{
			// conservative padding, like TBasicTriangle::getAABB's epsilon (TBasicTriangle.ipp)
			const float pad = 1e-4f + 1e-6f * std::max(std::abs(nd.lo[a]), std::abs(nd.hi[a]));
			nd.lo[a] -= pad; nd.hi[a] += pad;
		}
		nd.begin = j.b;
		nd.count = j.e - j.b;
		if(nd.count <= 2)
		{
			continue;
		}
		int axis = 0;
		float ext = -1;
		for(int a = 0; a < 3; ++a) { if(nd.hi[a] - nd.lo[a] > ext) { ext = nd.hi[a] - nd.lo[a]; axis = a; } }
		const uint32_t mid = (j.b + j.e) / 2;
		std::nth_element(s.order.begin() + j.b, s.order.begin() + mid, s.order.begin() + j.e,
			[&](uint32_t x, uint32_t y) { return cen[3 * x + axis] < cen[3 * y + axis]; });
		const int l = static_cast<int>(s.nodes.size());
		s.nodes.push_back(Node{});
		s.nodes.push_back(Node{});
		s.nodes[j.node].left = l;
		s.nodes[j.node].right = l + 1;
		s.nodes[j.node].count = 0;
		stack.push_back({l, j.b, mid});
		stack.push_back({l + 1, mid, j.e});
	}
}

// TAABB3D::intersectVolumeRobust (Math/Geometry/TAABB3D.ipp:391-420), including its handling of
// negative-zero direction components (treated as positive, so such rays miss boxes they start in).
bool box_hit(const Node& nd, Vec o, Vec d, Vec inv, float t0, float t1)
{
	const float oo[3] = {o.x, o.y, o.z}, ii[3] = {inv.x, inv.y, inv.z}, dd[3] = {d.x, d.y, d.z};
	for(int a = 0; a < 3; ++a)
	{
		const float slab[2] = {nd.lo[a] - oo[a], nd.hi[a] - oo[a]};
		const bool neg = dd[a] < 0;
		const float mn = slab[neg] * ii[a];
		const float mx = slab[1 - neg] * ii[a];
		t0 = mn > t0 ? mn : t0;
		t1 = mx < t1 ? mx : t1;
	}
	return t0 <= t1 * (std::numeric_limits<float>::epsilon() * 2 + 1);
}

// Closest hit (TBinaryBvhIntersector::isIntersecting) or any hit (isOccluding) over all triangles.
bool trace(const Scene& s, Vec o, Vec d, float tmin, float tmax, bool any, int* out_tri, float* out_t, float b[3])
{
	const Vec inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
	int best = -1;
	float best_t = tmax;
	float bb[3] = {0, 0, 0};
	int stack[256];
	int sp = 0;
	stack[sp++] = 0;
	while(sp)
	{
		const Node& nd = s.nodes[stack[--sp]];
		if(!box_hit(nd, o, d, inv, tmin, best_t))
		{
			continue;
		}
		if(nd.left < 0)
		{
			for(uint32_t i = nd.begin; i < nd.begin + nd.count; ++i)
			{
				const uint32_t k = s.order[i];
				const Tri& t = s.tris[k];
				float th, bc[3];
				if(watertight(o, d, tmin, best_t, t.a, t.b, t.c, &th, bc))
				{
					if(any)
					{
						return true;
					}
					if(th < best_t || static_cast<int>(k) < best)
					{
						best = static_cast<int>(k);
						best_t = th;
						bb[0] = bc[0]; bb[1] = bc[1]; bb[2] = bc[2];
					}
				}
			}
		}
		else if(sp < 254)
		{
			stack[sp++] = nd.left;
			stack[sp++] = nd.right;
		}
	}
	if(best < 0)
	{
		return false;
	}
	*out_tri = best;
	*out_t = best_t;
	b[0] = bb[0]; b[1] = bb[1]; b[2] = bb[2];
	return true;
}

// ----------------------------------------------------------------------------------------------
// Surface frames and BSDFs.

struct Surface
{
	Vec pos, ng, ns, bx, bz;    // shading basis: bx, ns, bz
	int tri = -1;
};

// PTriangle face normal (PTriangle.cpp:19-35) and Basis3R::makeFromUnitY (TOrthonormalBasis3.ipp:16-39)
Vec face_normal(const Tri& t)
{
	const Vec n = cross(t.b - t.a, t.c - t.a);
	const float l2 = dot(n, n);
	if(!(l2 > 0) || std::isinf(l2))
	{
		return mk(0, 1, 0);
	}
	return unit(n);
}

void make_basis(Surface& x)
{
	const Vec n = x.ns;
	Vec bx;
	if(std::abs(n.y) < 0.70710678118654752f)
	{
		bx = mk(-n.z, 0, n.x);
		bx = bx * (1.0f / std::sqrt(bx.x * bx.x + bx.z * bx.z));
	}
	else
	{
		bx = mk(n.y, -n.x, 0);
		bx = bx * (1.0f / std::sqrt(bx.x * bx.x + bx.y * bx.y));
	}
	x.bx = bx;
	x.bz = cross(bx, n);
}

// Strict sidedness (Core/LTA/SidednessAgreement.h:119-280)
bool agreed(const Surface& x, Vec v) { return dot(x.ng, v) * dot(x.ns, v) > 0; }
bool same_hemi(const Surface& x, Vec a, Vec b) { return agreed(x, a) && agreed(x, b) && dot(a, x.ng) * dot(b, x.ng) > 0; }
bool opp_hemi(const Surface& x, Vec a, Vec b) { return agreed(x, a) && agreed(x, b) && dot(a, x.ng) * dot(b, x.ng) < 0; }

// IsoTrowbridgeReitz (Core/SurfaceBehavior/Property/IsoTrowbridgeReitz.cpp:20-56) and the
// height-correlated masking-shadowing of ShapeInvariantMicrofacet.cpp:20-70.
float ggx_lambda(float alpha, Vec n, Vec w)
{
	const float nd = dot(n, w);
	const float nd2 = std::min(nd * nd, 1.0f);
	return 0.5f * (-1.0f + std::sqrt(1.0f + alpha * alpha * (1.0f / nd2 - 1.0f)));
}
float ggx_d(float alpha, Vec n, Vec h)
{
	const float noh = dot(n, h);
	const float a2 = alpha * alpha;
	const float inner = noh * noh * (a2 - 1.0f) + 1.0f;
	return a2 / (kPi * inner * inner);
}
float ggx_g(float alpha, Vec n, Vec h, Vec l, Vec v)
{
	const float nol = dot(n, l), nov = dot(n, v), hol = dot(h, l), hov = dot(h, v);
	if(!(hol * nol > 0 && hov * nov > 0))
	{
		return 0;
	}
	return 1.0f / (1.0f + ggx_lambda(alpha, n, l) + ggx_lambda(alpha, n, v));
}
float ggx_vndf(float alpha, Vec n, Vec h, Vec v)
{
	const float g1 = 1.0f / (1.0f + ggx_lambda(alpha, n, v));
	return g1 * ggx_d(alpha, n, h) * std::abs(dot(h, v) / dot(n, v));
}
// TrowbridgeReitz::sampleVisibleH (TrowbridgeReitz.cpp:19-82)
Vec ggx_sample_h(const Surface& x, float alpha, Vec v, float u0, float u1)
{
	const Vec up = dot(v, x.ns) >= 0 ? v : -v;
	const Vec lv = mk(dot(x.bx, up), dot(x.ns, up), dot(x.bz, up));
	const Vec sv = unit(mk(lv.x * alpha, lv.y, lv.z * alpha));
	const float phi = 2 * kPi * u0;
	const float y = std::fma(1.0f - u1, 1.0f + sv.y, -sv.y);
	const float st = std::sqrt(std::min(std::max(1.0f - y * y, 0.0f), 1.0f));
	const Vec hemi = mk(st * std::sin(phi), y, st * std::cos(phi)) + sv;
	const Vec lh = mk(hemi.x * alpha, hemi.y, hemi.z * alpha);
	const Vec wh = x.bx * lh.x + x.ns * lh.y + x.bz * lh.z;
	const float l2 = dot(wh, wh);
	const Vec h = wh * (1.0f / std::sqrt(l2));
	return (l2 > 0 && std::isfinite(h.x) && std::isfinite(h.y) && std::isfinite(h.z)) ? h : x.ns;
}
bool half_same(Vec l, Vec v, Vec n, Vec* h)
{
	Vec s = l + v;
	if(is_zero(s)) { return false; }
	s = unit(s);
	const float nh = dot(n, s);
	s = s * (nh > 0 ? 1.0f : (nh < 0 ? -1.0f : 0.0f));
	*h = s;
	return !is_zero(s);
}
// SchlickApproxConductorFresnel.cpp:35-40 (std::pow(float, int) evaluates in double)
Rgb schlick(Rgb f0, float c)
{
	const float m = static_cast<float>(std::pow(static_cast<double>(1.0f - std::abs(c)), 5));
	return Rgb{(1 - f0.r) * m + f0.r, (1 - f0.g) * m + f0.g, (1 - f0.b) * m + f0.b};
}
// ExactDielectricFresnel.cpp:12-40
float fresnel_d(float eo, float ei, float ci)
{
	float eta_i = eo, eta_t = ei;
	if(ci < 0) { std::swap(eta_i, eta_t); ci = std::abs(ci); }
	const float r = eta_i / eta_t;
	const float st2 = (1 - ci * ci) * r * r;
	if(st2 >= 1) { return 1; }
	const float ct = std::sqrt(1 - st2);
	const float rp = (eta_t * ci - eta_i * ct) / (eta_t * ci + eta_i * ct);
	const float rs = (eta_i * ci - eta_t * ct) / (eta_i * ci + eta_t * ct);
	return 0.5f * (rp * rp + rs * rs);
}
float reflect_prob(float f) { return std::min(std::max(f, 0.0001f), 1.0f - 0.0001f); }

// SurfaceOptics::calcBsdf + the three optics' calcBsdf
bool bsdf_eval(const Material& m, const Surface& x, Vec l, Vec v, Rgb* out)
{
	if(!agreed(x, l) || !agreed(x, v)) { return false; }
	const Vec n = x.ns;
	if(m.type == 0)
	{
		if(!same_hemi(x, l, v)) { return false; }
		*out = m.c * (1.0f / kPi);
		return true;
	}
	if(m.type == 1)
	{
		if(!same_hemi(x, l, v)) { return false; }
		Vec h;
		if(!half_same(l, v, n, &h)) { return false; }
		*out = schlick(m.c, dot(h, l)) * (ggx_d(m.alpha, n, h) * ggx_g(m.alpha, n, h, l, v) / (4 * std::abs(dot(n, v) * dot(n, l))));
		return finite(*out);
	}
	const float nol = dot(n, l), nov = dot(n, v);
	if(nol * nov == 0) { return false; }
	if(same_hemi(x, l, v))
	{
		Vec h;
		if(!half_same(l, v, n, &h)) { return false; }
		const float f = fresnel_d(m.ior_outer, m.ior_inner, dot(h, l)) *
			(ggx_d(m.alpha, n, h) * ggx_g(m.alpha, n, h, l, v) / (4 * std::abs(nol * nov)));
		*out = Rgb{f, f, f};
		return std::isfinite(f);
	}
	if(opp_hemi(x, l, v))
	{
		float ei = m.ior_outer, et = m.ior_inner;
		if(nol < 0) { std::swap(ei, et); }
		Vec h = l * (-ei) + v * (-et);
		if(is_zero(h)) { return false; }
		h = unit(h);
		if(dot(n, h) < 0) { h = -h; }
		const float hov = dot(h, v), hol = dot(h, l);
		const float F = 1 - fresnel_d(m.ior_outer, m.ior_inner, hol);
		const float ior_term = (et / ei) * ei / (ei * hol + et * hov);
		if(!std::isfinite(ior_term)) { return false; }
		const float f = F * (ggx_d(m.alpha, n, h) * ggx_g(m.alpha, n, h, l, v) * std::abs(hol * hov / (nol * nov)) * (ior_term * ior_term));
		*out = Rgb{f, f, f};
		return std::isfinite(f);
	}
	return false;
}

// SurfaceOptics::calcBsdfPdf + the three optics' calcBsdfPdf; 0 = empty/invalid
float bsdf_pdf(const Material& m, const Surface& x, Vec l, Vec v)
{
	if(!agreed(x, l) || !agreed(x, v)) { return 0; }
	const Vec n = x.ns;
	float p = 0;
	if(m.type == 0)
	{
		if(!same_hemi(x, l, v)) { return 0; }
		p = std::abs(dot(l, n)) * (1.0f / kPi);
	}
	else if(m.type == 1)
	{
		if(!same_hemi(x, l, v)) { return 0; }
		Vec h;
		if(!half_same(l, v, n, &h)) { return 0; }
		p = ggx_vndf(m.alpha, n, h, v) / (4 * std::abs(dot(h, l)));
	}
	else if(same_hemi(x, l, v))
	{
		Vec h;
		if(!half_same(l, v, n, &h)) { return 0; }
		p = ggx_vndf(m.alpha, n, h, v) / (4 * std::abs(dot(h, l))) * reflect_prob(fresnel_d(m.ior_outer, m.ior_inner, dot(h, l)));
	}
	else if(opp_hemi(x, l, v))
	{
		float ei = m.ior_outer, et = m.ior_inner;
		if(dot(n, l) < 0) { std::swap(ei, et); }
		Vec h = l * (-ei) + v * (-et);
		if(is_zero(h)) { return 0; }
		h = unit(h);
		if(dot(n, h) < 0) { h = -h; }
		const float hov = dot(h, v), hol = dot(h, l);
		const float it = ei * hol + et * hov;
		p = ggx_vndf(m.alpha, n, h, v) * (std::abs(ei * ei * hol) / (it * it)) *
			(1 - reflect_prob(fresnel_d(m.ior_outer, m.ior_inner, hol)));
	}
	return (std::isfinite(p) && p > 0) ? p : 0;
}

struct Sample
{
	Vec l;
	Rgb w;
	float rel_ior = 1;
	bool ok = false;
};

// SurfaceOptics::genBsdfSample + the three optics' genBsdfSample
Sample bsdf_sample(const Material& m, const Surface& x, Vec v, float u0, float u1, float u2)
{
	Sample s;
	if(!agreed(x, v)) { return s; }
	const Vec n = x.ns;
	if(m.type == 0)
	{
		// THemisphere::sampleToSurfaceCosThetaWeighted (Math/Geometry/THemisphere.h:104-120)
		const float phi = 2 * kPi * u0, yv = std::sqrt(u1), yr = std::sqrt(1 - yv * yv);
		const Vec loc = mk(std::sin(phi) * yr, yv, std::cos(phi) * yr);
		Vec l = unit(x.bx * loc.x + x.ns * loc.y + x.bz * loc.z);
		if(dot(v, n) < 0) { l = -l; }
		s.l = l;
		s.w = m.c;
	}
	else if(m.type == 1)
	{
		const Vec h = ggx_sample_h(x, m.alpha, v, u0, u1);
		const Vec mv = -v;
		const Vec l = unit(mv - h * (2 * dot(h, mv)));
		const float hol = dot(h, l);
		s.l = l;
		s.w = schlick(m.c, hol) * (ggx_g(m.alpha, n, h, l, v) * ggx_d(m.alpha, n, h) * std::abs(hol / dot(n, v)) / ggx_vndf(m.alpha, n, h, v));
	}
	else
	{
		const Vec h = ggx_sample_h(x, m.alpha, v, u0, u1);
		const float fr = fresnel_d(m.ior_outer, m.ior_inner, dot(h, v));
		const float rp = reflect_prob(fr);
		float F;
		Vec l;
		if(u2 < rp)
		{
			const Vec mv = -v;
			l = unit(mv - h * (2 * dot(h, mv)));
			if(!same_hemi(x, v, l)) { return s; }
			F = fr / rp;
		}
		else
		{
			// DielectricFresnel::calcRefractDir (DielectricFresnel.cpp:18-42)
			const float ion = dot(v, h);
			const float sgn = ion < 0 ? -1.0f : 1.0f;
			const float ratio = sgn < 0 ? m.ior_inner / m.ior_outer : m.ior_outer / m.ior_inner;
			const float sq = 1 - ratio * ratio * (1 - ion * ion);
			if(sq <= 0) { return s; }
			l = unit(h * (ratio * ion - sgn * std::sqrt(sq)) + v * (-ratio));
			if(!opp_hemi(x, v, l)) { return s; }
			F = 1 - fresnel_d(m.ior_outer, m.ior_inner, dot(h, l));
			float ei = m.ior_outer, et = m.ior_inner;
			if(dot(n, l) < 0) { std::swap(ei, et); }
			s.rel_ior = et / ei;
			F *= s.rel_ior * s.rel_ior;
			F /= (1 - rp);
		}
		const float val = F * (ggx_g(m.alpha, n, h, l, v) * ggx_d(m.alpha, n, h) * std::abs(dot(h, v) / dot(n, v)) / ggx_vndf(m.alpha, n, h, v));
		s.l = l;
		s.w = Rgb{val, val, val};
	}
	const float c = std::abs(dot(n, s.l));
	s.ok = finite(s.w) && c > 0 && c < 1.1f && agreed(x, s.l);
	return s;
}

// ----------------------------------------------------------------------------------------------
// SurfaceHitRefinery iterative offsets (Core/LTA/SurfaceHitRefinery.cpp:62-263).

bool reint(const Tri& t, Vec o, Vec d, float tmin, float tmax, float* th)
{
	float b[3];
	return watertight(o, d, tmin, tmax, t.a, t.b, t.c, th, b);
}

struct Offset
{
	Vec offset, dir;
	float max_distance;
};

Offset offset_from(const Surface& x, const Tri& tri, Vec dir)
{
	const Vec od = dot(x.ng, dir) > 0 ? x.ng : -x.ng;
	const Vec ed = unit(dir);
	const float ec = std::min(std::max(dot(ed, od), 0.0f), 1.0f);
	// HitDetail stores the triangle's error factors (5e-8, 2.5e-5) as powers of two, 2^-24 and 2^-15
	// (Core/HitDetail.h:185-200)
	float mx = len(x.pos) * 5.9604644775390625e-8f + std::numeric_limits<float>::min(), mn = 0;
	for(int it = 0; it < 64; ++it)
	{
		float t;
		if(!reint(tri, x.pos + od * mx, ed, 0, kFltMax, &t)) { break; }
		mx += t * ec;
		mn = mx;
		mx *= 2;
	}
	for(int it = 0, refine = 0; refine < 1 && it < 64; ++it)
	{
		const float mid = (mn + mx) * 0.5f;
		if(!(mn < mid && mid < mx)) { break; }
		float t;
		if(!reint(tri, x.pos + od * mid, ed, 0, kFltMax, &t)) { mx = mid; ++refine; }
		else { mn = std::min(std::max(mid + t * ec, mid), mx); }
	}
	return Offset{od * mx, ed, kFltMax};
}

Offset mutual_offset(const Surface& x, const Tri& tri, Vec pos2, const Tri& tri2)
{
	const Offset r = offset_from(x, tri, pos2 - x.pos);
	const float init = len(pos2) * 3.0517578125e-5f + std::numeric_limits<float>::min();
	const Vec origin = x.pos + r.offset;
	const float dist = len(origin - pos2);
	float mx = init, mn = 0;
	for(int it = 0; it < 64 && dist > mx; ++it)
	{
		float t;
		if(!reint(tri2, origin, r.dir, 0, dist - mx, &t)) { break; }
		mx = std::max(dist - t, mx);
		mn = mx;
		mx *= 2;
	}
	for(int it = 0, refine = 0; dist > mx && refine < 1 && it < 64; ++it)
	{
		const float mid = (mn + mx) * 0.5f;
		if(!(mn < mid && mid < mx)) { break; }
		float t;
		if(!reint(tri2, origin, r.dir, 0, dist - mid, &t)) { mx = mid; ++refine; }
		else { mn = std::min(std::max(dist - t, mid), mx); }
	}
	return Offset{r.offset, r.dir, std::max(dist - mx, 0.0f)};
}

// ----------------------------------------------------------------------------------------------
// Random numbers: a PCG32 stream per worker (Math/Random/Random.cpp:25-44 uses thread-local PCG32).

struct Pcg32
{
	uint64_t state, inc;
	explicit Pcg32(uint64_t seed, uint64_t seq = 0x853c49e6748fea9bull) : state(0), inc((seq << 1) | 1) { next(); state += seed; next(); }
	uint32_t next()
	{
		const uint64_t old = state;
		state = old * 6364136223846793005ull + inc;
		const uint32_t xs = static_cast<uint32_t>(((old >> 18) ^ old) >> 27);
		const uint32_t rot = static_cast<uint32_t>(old >> 59);
		return (xs >> rot) | (xs << ((-rot) & 31));
	}
	float u01() { return static_cast<float>(next() >> 8) * (1.0f / 16777216.0f); }
};

float lum(Rgb c) { return 0.212639004f * c.r + 0.715168655f * c.g + 0.0721923187f * c.b; }

// pdfA_to_pdfW (Core/LTA/lta.h:17-25)
float pdfa_to_w(float pdfa, Vec to_target, Vec n)
{
	const float d2 = dot(to_target, to_target);
	const float w = pdfa / dot(unit(to_target), n) * d2;
	return std::isfinite(w) ? std::abs(w) : 0;
}

float tri_area(const Tri& t) { return len(cross(t.b - t.a, t.c - t.a)) * 0.5f; }

bool surface_at(const Scene& s, Vec o, Vec d, Surface* x, Vec* dir_in)
{
	int k;
	float t, b[3];
	if(!trace(s, o, d, 0, kFltMax, false, &k, &t, b))
	{
		return false;
	}
	const Tri& tr = s.tris[k];
	x->pos = tr.a * b[0] + tr.b * b[1] + tr.c * b[2];
	x->ng = face_normal(tr);
	x->ns = x->ng;
	x->tri = k;
	make_basis(*x);
	*dir_in = d;
	return true;
}

// ---- the dome (Core/Emitter/LatLongEnvEmitter.cpp:36-150, Core/Intersection/PLatLongEnvSphere.cpp)

struct EnvConfig
{
	std::vector<float> rgb;
	uint32_t w = 0, h = 0;
	double rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
	double center[3] = {0, 0, 0};
	bool exact = false;
};

EnvConfig& env_config()
{
	static EnvConfig cfg;
	return cfg;
}

// Lat-long coordinates of a world direction (TSphere::surfaceToLatLong01 in the dome's frame).
void env_uv(const Scene& s, Vec d, double* u, double* v)
{
	const double* R = s.env_rot;
	const double lx = R[0] * d.x + R[3] * d.y + R[6] * d.z;
	const double ly = R[1] * d.x + R[4] * d.y + R[7] * d.z;
	const double lz = R[2] * d.x + R[5] * d.y + R[8] * d.z;
	const double len = std::sqrt(lx * lx + ly * ly + lz * lz);
	const double theta = std::acos(std::min(std::max(len > 0 ? ly / len : 1.0, -1.0), 1.0));
	double phi = std::atan2(lx, lz);
	if(phi < 0) { phi += 2 * M_PI; }
	*u = phi / (2 * M_PI);
	*v = (M_PI - theta) / M_PI;
}

// Bilinear with clamped edges (TPixelTexture2D::samplePixelBufferBilinear).
Rgb env_lookup(const Scene& s, double u, double v)
{
	const int w = static_cast<int>(s.env_w), h = static_cast<int>(s.env_h);
	const double x = std::min(std::max(u, 0.0), 1.0) * w - 0.5, y = std::min(std::max(v, 0.0), 1.0) * h - 0.5;
	const double fx = std::floor(x), fy = std::floor(y), ax = x - fx, ay = y - fy;
	auto at = [&](int i, int j)
	{
		i = std::min(std::max(i, 0), w - 1);
		j = std::min(std::max(j, 0), h - 1);
		return s.env_texels[static_cast<std::size_t>(j) * w + i];
	};
	const int i0 = static_cast<int>(fx), j0 = static_cast<int>(fy);
	return at(i0, j0) * static_cast<float>((1 - ax) * (1 - ay)) + at(i0, j0 + 1) * static_cast<float>((1 - ax) * ay) +
	       at(i0 + 1, j0) * static_cast<float>(ax * (1 - ay)) + at(i0 + 1, j0 + 1) * static_cast<float>(ax * ay);
}

double env_distance(const Scene& s, Vec x, Vec w)
{
	const double ox = x.x - s.env_center[0], oy = x.y - s.env_center[1], oz = x.z - s.env_center[2];
	const double b = ox * w.x + oy * w.y + oz * w.z;
	const double c = ox * ox + oy * oy + oz * oz - s.env_radius * s.env_radius;
	return -b + std::sqrt(std::max(b * b - c, 0.0));
}

double env_texel_pdf(const Scene& s, double u, double v)
{
	const uint32_t i = std::min(static_cast<uint32_t>(std::max(u, 0.0) * s.env_w), s.env_w - 1);
	const uint32_t j = std::min(static_cast<uint32_t>(std::max(v, 0.0) * s.env_h), s.env_h - 1);
	return s.env_pdf_uv[static_cast<std::size_t>(j) * s.env_w + i];
}

// Solid-angle density the reference assigns to a BSDF-sampled ray from x along w that leaves
// the scene (LatLongEnvEmitter::calcDirectPdf: area density on the dome sphere, converted with
// the distance and cosine at the ray's hit on it), or the exact density.
double env_pdf_hit(const Scene& s, Vec x, Vec w)
{
	double u, v;
	env_uv(s, w, &u, &v);
	double pdf = env_texel_pdf(s, u, v) / (2 * M_PI * M_PI * std::sin(M_PI * (1 - v)));
	if(!s.env_exact)
	{
		const double d = env_distance(s, x, w);
		const double px = x.x + d * w.x - s.env_center[0], py = x.y + d * w.y - s.env_center[1], pz = x.z + d * w.z - s.env_center[2];
		const double cos_p = std::abs(px * w.x + py * w.y + pz * w.z) / s.env_radius;
		pdf *= d * d / (s.env_radius * s.env_radius * cos_p);
	}
	return std::isfinite(pdf) && pdf > 0 ? pdf : 0;
}

// A dome sample for NEE at x (LatLongEnvEmitter::genDirectSample with
// PLatLongEnvSphere::genPosSampleWithObservationPos): uv from the 2D piecewise-constant
// distribution, its direction w, the reference's density (the cosine at the end of an observation
// ray of length r, projected onto the sphere, where the shadow ray also aims) or the exact one.
bool env_sample(const Scene& s, Vec x, float r0, float r1, Vec* w_out, double* pdf_out, Rgb* le, Vec* shadow_dir)
{
	const std::size_t h = s.env_h, wdt = s.env_w;
	std::size_t j = std::min<std::size_t>(std::upper_bound(s.env_row_cdf.begin() + 1, s.env_row_cdf.end(), r0) -
	                                      (s.env_row_cdf.begin() + 1), h - 1);
	const double rj0 = s.env_row_cdf[j], rj1 = s.env_row_cdf[j + 1];
	const double fv = rj1 > rj0 ? (r0 - rj0) / (rj1 - rj0) : 0.5;
	const double* col = &s.env_col_cdf[j * (wdt + 1)];
	std::size_t i = std::min<std::size_t>(std::upper_bound(col + 1, col + wdt + 1, r1) - (col + 1), wdt - 1);
	const double fu = col[i + 1] > col[i] ? (r1 - col[i]) / (col[i + 1] - col[i]) : 0.5;
	const double u = (i + std::min(std::max(fu, 0.0), 1.0)) / wdt, v = (j + std::min(std::max(fv, 0.0), 1.0)) / h;
	const double theta = (1 - v) * M_PI, phi = 2 * M_PI * u, st = std::sin(theta);
	const double lx = st * std::sin(phi), ly = std::cos(theta), lz = st * std::cos(phi);
	const double* R = s.env_rot;
	const Vec w = mk(static_cast<float>(R[0] * lx + R[1] * ly + R[2] * lz), static_cast<float>(R[3] * lx + R[4] * ly + R[5] * lz),
	                 static_cast<float>(R[6] * lx + R[7] * ly + R[8] * lz));
	double pdf = s.env_pdf_uv[j * wdt + i] / (2 * M_PI * M_PI * st);
	Vec sd = w;
	if(!s.env_exact)
	{
		const double d = env_distance(s, x, w);
		double qx = x.x + s.env_radius * w.x - s.env_center[0], qy = x.y + s.env_radius * w.y - s.env_center[1],
		       qz = x.z + s.env_radius * w.z - s.env_center[2];
		const double ql = std::sqrt(qx * qx + qy * qy + qz * qz);
		qx /= ql; qy /= ql; qz /= ql;
		pdf *= d * d / (s.env_radius * s.env_radius * std::abs(qx * w.x + qy * w.y + qz * w.z));
		sd = mk(static_cast<float>(s.env_center[0] + s.env_radius * qx - x.x), static_cast<float>(s.env_center[1] + s.env_radius * qy - x.y),
		        static_cast<float>(s.env_center[2] + s.env_radius * qz - x.z));
	}
	if(!(st > 0) || !std::isfinite(pdf) || !(pdf > 0)) { return false; }
	*w_out = w;
	*pdf_out = pdf;
	*le = env_lookup(s, u, v);
	*shadow_dir = sd;
	return true;
}

// One path of BNEEPTEstimator::estimate (Core/Estimator/BNEEPTEstimator.cpp:38-262),
// BVPTEstimator::estimate (Core/Estimator/BVPTEstimator.cpp:25-160) or
// BVPTDLEstimator::estimate (Core/Estimator/BVPTDLEstimator.cpp:21-96): BVPT cut after one
// BSDF-sampled bounce, with the emitted radiance rather than the path weight clamped.
Rgb estimate(const Scene& s, Vec o, Vec d, uint32_t max_bounces, Pcg32& rng)
{
	const bool bvpt = s.estimator == 1 || s.estimator == 2;
	const bool dl = s.estimator == 2;
	if(dl) { max_bounces = 1; }
	Rgb energy;
	Rgb thr{1, 1, 1};
	float rr_scale = 1;
	Surface x;
	Vec din;
	auto env_hit = [&](Vec dir, Rgb* le)
	{
		if(s.env < 0) { return false; }
		double u, v;
		env_uv(s, dir, &u, &v);
		*le = env_lookup(s, u, v);
		return true;
	};
	if(!surface_at(s, o, d, &x, &din))
	{
		Rgb le;
		if(env_hit(d, &le)) { energy = energy + le; }
		return energy;
	}
	if(!(dot(x.ng, d) * dot(x.ns, d) > 0)) { return energy; }
	auto emitted = [&](const Surface& xe, Vec dir, Rgb* le) -> int
	{
		const uint32_t e = s.tris[xe.tri].emitter;
		if(!e) { return -1; }
		*le = dot(-dir, xe.ns) > 0 ? s.emitters[e - 1].radiance : Rgb{};
		return static_cast<int>(e - 1);
	};
	{
		Rgb le;
		if(emitted(x, d, &le) >= 0) { energy = energy + le; }
	}
	for(uint32_t bounce = 0; bounce < max_bounces; ++bounce)
	{
		const Material& m = s.materials[s.tris[x.tri].material];
		const Vec v = -d;
		// NEE (TDirectLightEstimator::neeSampleEmission, TDirectLightEstimator.ipp:71-102)
		if(!bvpt && !s.emitters.empty() && m.type != 3)
		{
			const float u = rng.u01();
			const std::size_t ei = std::min<std::size_t>(
				std::upper_bound(s.cdf.begin(), s.cdf.end(), u) - s.cdf.begin(), s.emitters.size() - 1);
			const Emitter& e = s.emitters[ei];
			Vec to_light;
			Rgb env_radiance_nee = e.radiance;
			float pdfw = 0;
			Offset vis{};
			bool ok = false;
			if(e.type == 1)
			{
				const float r0 = rng.u01(), r1 = rng.u01();
				double env_pdf = 0;
				Vec shadow_dir;
				Rgb env_le;
				if(env_sample(s, x.pos, r0, r1, &to_light, &env_pdf, &env_le, &shadow_dir) && agreed(x, to_light))
				{
					pdfw = static_cast<float>(e.pmf * env_pdf);
					env_radiance_nee = env_le;
					vis = offset_from(x, s.tris[x.tri], shadow_dir);
					ok = pdfw > 0;
				}
			}
			else if(!e.tris.empty())
			{
				const Tri& lt = s.tris[e.tris[std::min<std::size_t>(static_cast<std::size_t>(rng.u01() * e.tris.size()), e.tris.size() - 1)]];
				const float A = std::sqrt(rng.u01()), B = rng.u01();
				const Vec xe = lt.a * (1 - A) + lt.b * (A * (1 - B)) + lt.c * (B * A);
				const Vec ne = face_normal(lt);
				const Vec e2t = x.pos - xe;
				if(dot(e2t, ne) > 0)
				{
					pdfw = pdfa_to_w(1 / tri_area(lt), e2t, ne) * (1.0f / e.tris.size()) * e.pmf;
					to_light = xe - x.pos;
					if(pdfw > 0 && std::isfinite(pdfw) && agreed(x, to_light))
					{
						vis = mutual_offset(x, s.tris[x.tri], xe, lt);
						ok = vis.max_distance > 0 && std::isfinite(vis.max_distance);
					}
				}
			}
			int k;
			float t, b[3];
			if(ok && !trace(s, x.pos + vis.offset, vis.dir, 0, vis.max_distance, true, &k, &t, b))
			{
				const Vec l = unit(to_light);
				Rgb f;
				if(bsdf_eval(m, x, l, v, &f))
				{
					const float pb = bsdf_pdf(m, x, l, v);
					const float mis = pdfw * pdfw / (pdfw * pdfw + pb * pb);
					Rgb w = f * std::abs(dot(x.ns, l));
					w = w * thr;
					w = w * (mis / pdfw);
					energy = energy + (e.type == 1 ? env_radiance_nee : e.radiance) * safe_clamp(w);
				}
			}
		}
		// BSDF sample + extension
		const Sample bs = bsdf_sample(m, x, v, rng.u01(), rng.u01(), rng.u01());
		if(!bs.ok) { break; }
		const Offset esc = offset_from(x, s.tris[x.tri], bs.l);
		const Vec no = x.pos + esc.offset;
		const Vec nd = esc.dir;
		Surface nx;
		Vec ndin;
		const bool hit = surface_at(s, no, nd, &nx, &ndin);
		if(hit && !(dot(nx.ng, nd) * dot(nx.ns, nd) > 0))
		{
			break;
		}
		const Rgb w_emit = thr * bs.w;
		Rgb le;
		int emitter = -1;
		bool have_le = false;
		if(hit) { emitter = emitted(nx, nd, &le); have_le = emitter >= 0; }
		else { have_le = env_hit(nd, &le); emitter = s.env; }
		if(have_le)
		{
			if(bvpt)
			{
				// BVPT adds emission with the post-roulette throughput, below
			}
			else if(!zero(le))
			{
				const float pb = bsdf_pdf(m, x, bs.l, v);
				if(pb > 0)
				{
					float lp = 0;
					const Emitter& e = s.emitters[emitter];
					if(e.type == 1) { lp = static_cast<float>(e.pmf * env_pdf_hit(s, x.pos, nd)); }
					else
					{
						const Vec tt = x.pos - nx.pos;
						if(dot(tt, nx.ns) > 0) { lp = pdfa_to_w(1 / tri_area(s.tris[nx.tri]), tt, nx.ns) * (1.0f / e.tris.size()) * e.pmf; }
					}
					const float mis = pb * pb / (pb * pb + lp * lp);
					energy = energy + le * safe_clamp(w_emit * mis);
				}
			}
		}
		thr = w_emit;
		rr_scale /= bs.rel_ior * bs.rel_ior;
		if(bounce >= 3)
		{
			const float surv = safe_clamp(lum(thr * rr_scale), 0, 0.95f);
			if(rng.u01() < surv) { thr = thr * (1.0f / surv); }
			else
			{
				break;
			}
		}
		if(bvpt && have_le)
		{
			energy = energy + (dl ? safe_clamp(le) * thr : le * safe_clamp(thr));
		}
		if(zero(thr) || !hit) { break; }
		x = nx;
		d = nd;
	}
	return energy;
}

}// end namespace port

// ----------------------------------------------------------------------------------------------
// Scene loading, rendering and the C ABI.

namespace
{

using namespace port;

Vec v3(const float* p) { return mk(p[0], p[1], p[2]); }

bool setup_scene(Scene& s, const float* cam, const float* tris, const uint32_t* tmat, const uint32_t* tem,
                 uint32_t n, const float* mats, uint32_t nm, const float* ems, uint32_t ne)
{
	s.tris.clear();
	for(uint32_t i = 0; i < n; ++i)
	{
		const float* t = tris + 9 * i;
		Tri tr{v3(t), v3(t + 3), v3(t + 6), tmat[i], tem ? tem[i] : 0u};
		// GTriangleMesh drops degenerate triangles (Actor/Geometry/GTriangleMesh.cpp:75-81)
		const Vec c = cross(tr.b - tr.a, tr.c - tr.a);
		const float l2 = dot(c, c);
		if(!(l2 > 0) || std::isinf(l2)) { continue; }
		s.tris.push_back(tr);
	}
	s.materials.clear();
	for(uint32_t i = 0; i < nm; ++i)
	{
		const float* p = mats + 8 * i;
		Material m{static_cast<int>(p[0]), Rgb{p[1], p[2], p[3]}, std::max(p[4] * p[4], 0.001f), p[5], p[6]};
		s.materials.push_back(m);
	}
	s.emitters.assign(ne, Emitter{});
	s.env = -1;
	for(uint32_t i = 0; i < ne; ++i)
	{
		s.emitters[i].radiance = Rgb{ems[4 * i], ems[4 * i + 1], ems[4 * i + 2]};
		s.emitters[i].type = static_cast<int>(ems[4 * i + 3]);
		if(s.emitters[i].type == 1) { s.env = static_cast<int>(i); s.env_radiance = s.emitters[i].radiance; }
	}
	double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
	for(uint32_t k = 0; k < s.tris.size(); ++k)
	{
		const Tri& t = s.tris[k];
		for(const Vec& v : {t.a, t.b, t.c})
		{
			lo[0] = std::min(lo[0], (double)v.x); hi[0] = std::max(hi[0], (double)v.x);
			lo[1] = std::min(lo[1], (double)v.y); hi[1] = std::max(hi[1], (double)v.y);
			lo[2] = std::min(lo[2], (double)v.z); hi[2] = std::max(hi[2], (double)v.z);
		}
		if(t.emitter) { s.emitters[t.emitter - 1].tris.push_back(k); }
	}
	// power-favouring pick (Core/Emitter/Sampler/ESPowerFavoring.cpp:21-49): luminance * area * pi
	// for triangle groups, luminance * dome area for the environment
	double total = 0;
	for(auto& e : s.emitters)
	{
		if(e.type == 1)
		{
			// the dome sphere around the scene bound (ADome.cpp:42-60) and its texel distribution
			// (LatLongEnvEmitter.cpp:52-79): weights max(luminance, 1e-6) * sin(theta) at texel centres
			const EnvConfig& cfg = env_config();
			std::copy(cfg.rot, cfg.rot + 9, s.env_rot);
			std::copy(cfg.center, cfg.center + 3, s.env_center);
			s.env_exact = cfg.exact;
			double r = 1;
			for(int c = 0; c < 8; ++c)
			{
				const double px = ((c & 1) ? hi[0] : lo[0]) - s.env_center[0], py = ((c & 2) ? hi[1] : lo[1]) - s.env_center[1];
				const double pz = ((c & 4) ? hi[2] : lo[2]) - s.env_center[2];
				r = std::max(r, std::sqrt(px * px + py * py + pz * pz) * 1.01);
			}
			s.env_radius = r;
			s.env_w = cfg.w ? cfg.w : 1;
			s.env_h = cfg.w ? cfg.h : 1;
			s.env_texels.clear();
			for(std::size_t k = 0; k < static_cast<std::size_t>(s.env_w) * s.env_h; ++k)
			{
				s.env_texels.push_back(cfg.w ? Rgb{cfg.rgb[3 * k], cfg.rgb[3 * k + 1], cfg.rgb[3 * k + 2]} : e.radiance);
			}
			std::vector<double> wts(s.env_texels.size());
			double sum = 0;
			for(uint32_t j = 0; j < s.env_h; ++j)
			{
				const double sin_theta = std::sin((1 - (j + 0.5) / s.env_h) * M_PI);
				for(uint32_t i = 0; i < s.env_w; ++i)
				{
					const std::size_t k = static_cast<std::size_t>(j) * s.env_w + i;
					wts[k] = std::max<double>(lum(s.env_texels[k]), 1e-6) * sin_theta;
					sum += wts[k];
				}
			}
			s.env_row_cdf.assign(s.env_h + 1, 0.0);
			s.env_col_cdf.assign(static_cast<std::size_t>(s.env_h) * (s.env_w + 1), 0.0);
			s.env_pdf_uv.assign(wts.size(), 0.0);
			for(uint32_t j = 0; j < s.env_h; ++j)
			{
				double row = 0;
				double* col = &s.env_col_cdf[static_cast<std::size_t>(j) * (s.env_w + 1)];
				for(uint32_t i = 0; i < s.env_w; ++i) { row += wts[static_cast<std::size_t>(j) * s.env_w + i]; col[i + 1] = row; }
				for(uint32_t i = 0; i <= s.env_w; ++i) { col[i] = row > 0 ? col[i] / row : (double)i / s.env_w; }
				s.env_row_cdf[j + 1] = s.env_row_cdf[j] + row / sum;
				for(uint32_t i = 0; i < s.env_w; ++i)
				{
					const std::size_t k = static_cast<std::size_t>(j) * s.env_w + i;
					s.env_pdf_uv[k] = wts[k] / sum * wts.size();
				}
			}
			e.weight = sum * 4 * M_PI * r * r;
		}
		else
		{
			double area = 0;
			for(uint32_t k : e.tris) { area += tri_area(s.tris[k]); }
			e.weight = std::max<double>(lum(e.radiance), 0) * area * M_PI;
		}
		total += e.weight;
	}
	s.cdf.clear();
	double acc = 0;
	for(auto& e : s.emitters)
	{
		e.pmf = total > 0 ? static_cast<float>(e.weight / total) : 0.0f;
		acc += e.weight;
		s.cdf.push_back(total > 0 ? static_cast<float>(acc / total) : 1.0f);
	}
	// camera (OrientedRasterObserver::makeRotFromVectors, SingleLensObserver::makeRasterToSensor)
	const Vec pos = v3(cam), dir = v3(cam + 3), up = v3(cam + 6);
	s.width = static_cast<uint32_t>(cam[10]);
	s.height = static_cast<uint32_t>(cam[11]);
	double z[3] = {-dir.x, -dir.y, -dir.z};
	const double zl = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
	for(double& c : z) { c /= zl; }
	double x[3] = {up.y * z[2] - up.z * z[1], up.z * z[0] - up.x * z[2], up.x * z[1] - up.y * z[0]};
	double y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]};
	const double xl = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]), yl = std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
	s.cam_pos = pos;
	s.ax = mk(x[0] / xl, x[1] / xl, x[2] / xl);
	s.ay = mk(y[0] / yl, y[1] / yl, y[2] / yl);
	s.az = mk(z[0], z[1], z[2]);
	s.sensor_w = 0.036f;
	s.sensor_h = static_cast<float>(0.036 / (static_cast<double>(s.width) / s.height));
	s.sensor_offset = static_cast<float>(0.018 / std::tan(cam[9] * M_PI / 180.0 * 0.5));
	build_bvh(s);
	return !s.tris.empty();
}

void render(const Scene& s, uint32_t spp, uint32_t max_bounces, uint32_t threads, uint64_t seed, double* sums)
{
	const uint32_t w = s.width, h = s.height;
	std::atomic<uint32_t> next_row{0};
	auto worker = [&](uint32_t wid)
	{
		Pcg32 rng(seed * 0x9E3779B97F4A7C15ull + wid + 1, wid * 2 + 1);
		std::vector<double> local;
		for(;;)
		{
			const uint32_t y = next_row.fetch_add(1);
			if(y >= h) { break; }
			for(uint32_t x = 0; x < w; ++x)
			{
				double acc[3] = {0, 0, 0};
				for(uint32_t k = 0; k < spp; ++k)
				{
					const float rx = x + rng.u01(), ry = y + rng.u01();
					const float sx = -s.sensor_w / w * rx + s.sensor_w * 0.5f;
					const float sy = -s.sensor_h / h * ry + s.sensor_h * 0.5f;
					const Vec recv = unit(s.ax * sx + s.ay * sy + s.az * s.sensor_offset);
					const Rgb e = estimate(s, s.cam_pos, -recv, max_bounces, rng);
					acc[0] += e.r; acc[1] += e.g; acc[2] += e.b;
				}
				double* p = sums + 3 * (static_cast<std::size_t>(y) * w + x);
				p[0] = acc[0]; p[1] = acc[1]; p[2] = acc[2];
			}
		}
	};
	std::vector<std::thread> pool;
	for(uint32_t t = 0; t < std::max(1u, threads); ++t) { pool.emplace_back(worker, t); }
	for(auto& t : pool) { t.join(); }
}

// Sample filters as the reference evaluates them, in FP64 (SampleFilter::make*, SampleFilter.cpp:
// 12-61: box 1 px; gaussian sigma 0.5, size 4, submerged by its value at (2, 2)
// (TGaussian2D.h); Mitchell-Netravali B = C = 1/3, size 4 (TMitchellNetravaliCubic2D.h:35-67);
// Blackman-Harris radius 2 (TBlackmanHarris2D.h:42-62)). 0 box, 1 gaussian, 2 mn, 3 bh.
double filter_half(int filter) { return filter == 0 ? 0.5 : 2.0; }

double filter_eval(int filter, double x, double y)
{
	if(filter == 1)
	{
		auto g = [](double a, double b) { return std::exp(-2.0 * a * a + -2.0 * b * b); };
		return std::max(g(x, y) - g(2.0, 2.0), 0.0);
	}
	if(filter == 2)
	{
		const double b = 1.0 / 3.0, c = 1.0 / 3.0;
		auto mn = [&](double v)
		{
			const double a = std::abs(v);
			if(a < 1) { return ((12 - 9 * b - 6 * c) * a * a * a + (-18 + 12 * b + 6 * c) * a * a + (6 - 2 * b)) / 6; }
			if(a < 2) { return ((-b - 6 * c) * a * a * a + (6 * b + 30 * c) * a * a + (-12 * b - 48 * c) * a + (8 * b + 24 * c)) / 6; }
			return 0.0;
		};
		return mn(x) * mn(y);
	}
	if(filter == 3)
	{
		auto bh = [](double v)
		{
			const double n = (v * 0.5 + 1.0) * 0.5;
			return 0.35875 - 0.48829 * std::cos(2 * M_PI * n) + 0.14128 * std::cos(4 * M_PI * n) -
			       0.01174 * std::cos(6 * M_PI * n);
		};
		return bh(x) * bh(y);
	}
	return 1.0;
}

// HdrRgbFilm::addRgbSample (HdrRgbFilm.cpp:82-123): the filter-weighted sample into every pixel
// whose centre lies within the filter's half size, and the weight into W; film [h][w][4].
void add_filtered_sample(double* film, uint32_t w, uint32_t h, int filter, double rx, double ry, const Rgb& e)
{
	const double half = filter_half(filter);
	const double fx0 = std::max(rx - half, 0.0), fy0 = std::max(ry - half, 0.0);
	const double fx1 = std::min(rx + half, static_cast<double>(w)), fy1 = std::min(ry + half, static_cast<double>(h));
	const int64_t x0 = static_cast<int64_t>(std::ceil(fx0 - 0.5)), y0 = static_cast<int64_t>(std::ceil(fy0 - 0.5));
	const int64_t x1 = static_cast<int64_t>(std::floor(fx1 - 0.5)) + 1, y1 = static_cast<int64_t>(std::floor(fy1 - 0.5)) + 1;
	for(int64_t y = y0; y < y1; ++y)
	{
		for(int64_t x = x0; x < x1; ++x)
		{
			const double f = filter_eval(filter, x - (rx - 0.5), y - (ry - 0.5));
			double* p = film + 4 * (static_cast<std::size_t>(y) * w + x);
			p[0] += e.r * f;
			p[1] += e.g * f;
			p[2] += e.b * f;
			p[3] += f;
		}
	}
}

// The render with a sample filter: samples spread uniformly over the film's sample window (the
// pixel-centre rectangle grown by the filter's half size, TSamplingFilm.ipp:102-119), one cell of
// it per pixel and sample, splatted into per-worker films that are summed at the end (the
// reference's per-worker films merged into the main film).
void render_filtered(const Scene& s, uint32_t spp, uint32_t max_bounces, uint32_t threads, uint64_t seed, int filter,
                     double* sums)
{
	const uint32_t w = s.width, h = s.height;
	const double half = filter_half(filter);
	const double wx0 = 0.5 - half, wy0 = 0.5 - half;
	const double cell_x = (w - 1 + 2 * half) / w, cell_y = (h - 1 + 2 * half) / h;
	const uint32_t nt = std::max(1u, threads);
	std::vector<std::vector<double>> films(nt, std::vector<double>(static_cast<std::size_t>(w) * h * 4, 0.0));
	std::atomic<uint32_t> next_row{0};
	auto worker = [&](uint32_t wid)
	{
		Pcg32 rng(seed * 0x9E3779B97F4A7C15ull + wid + 1, wid * 2 + 1);
		double* film = films[wid].data();
		for(;;)
		{
			const uint32_t y = next_row.fetch_add(1);
			if(y >= h) { break; }
			for(uint32_t x = 0; x < w; ++x)
			{
				for(uint32_t k = 0; k < spp; ++k)
				{
					const double rx = wx0 + (x + static_cast<double>(rng.u01())) * cell_x;
					const double ry = wy0 + (y + static_cast<double>(rng.u01())) * cell_y;
					const float sx = -s.sensor_w / w * static_cast<float>(rx) + s.sensor_w * 0.5f;
					const float sy = -s.sensor_h / h * static_cast<float>(ry) + s.sensor_h * 0.5f;
					const Vec recv = unit(s.ax * sx + s.ay * sy + s.az * s.sensor_offset);
					const Rgb e = estimate(s, s.cam_pos, -recv, max_bounces, rng);
					add_filtered_sample(film, w, h, filter, rx, ry, e);
				}
			}
		}
	};
	std::vector<std::thread> pool;
	for(uint32_t t = 0; t < nt; ++t) { pool.emplace_back(worker, t); }
	for(auto& t : pool) { t.join(); }
	std::fill(sums, sums + static_cast<std::size_t>(w) * h * 4, 0.0);
	for(const auto& f : films)
	{
		for(std::size_t i = 0; i < f.size(); ++i) { sums[i] += f[i]; }
	}
}

}// end anonymous namespace

extern "C" {

// The dome of the next renders: a lat-long image [h][w][3] (row 0 = bottom) with its rotation
// (row-major, dome local -> world) and centre; w = 0 keeps the emitter's constant radiance as a
// 1 x 1 image. exact != 0 uses the true densities instead of the reference's.
int port_set_environment(const float* rgb, uint32_t w, uint32_t h, const float* rot, const float* center, uint32_t exact)
{
	EnvConfig& cfg = env_config();
	cfg.w = rgb && w && h ? w : 0;
	cfg.h = rgb && w && h ? h : 0;
	cfg.rgb.assign(rgb && w && h ? rgb : nullptr, rgb && w && h ? rgb + static_cast<std::size_t>(w) * h * 3 : nullptr);
	for(int k = 0; k < 9; ++k) { cfg.rot[k] = rot ? rot[k] : (k % 4 == 0 ? 1.0 : 0.0); }
	for(int k = 0; k < 3; ++k) { cfg.center[k] = center ? center[k] : 0.0; }
	cfg.exact = exact != 0;
	return 0;
}

// Closest hit / occlusion over host triangles: rays [n][8] = origin, minT, direction, maxT.
int port_trace(const float* tris, uint32_t num_tris, const float* rays, uint32_t n,
               int32_t* out_prim, float* out_t, float* out_bary, int32_t* out_occluded)
{
	Scene s;
	for(uint32_t i = 0; i < num_tris; ++i)
	{
		const float* t = tris + 9 * i;
		s.tris.push_back(Tri{v3(t), v3(t + 3), v3(t + 6), 0, 0});
	}
	build_bvh(s);
	for(uint32_t i = 0; i < n; ++i)
	{
		const float* r = rays + 8 * i;
		int k;
		float t, b[3];
		const bool hit = trace(s, v3(r), v3(r + 4), r[3], r[7], false, &k, &t, b);
		out_prim[i] = hit ? k : -1;
		out_t[i] = hit ? t : 0;
		for(int c = 0; c < 3; ++c) { out_bary[3 * i + c] = hit ? b[c] : 0; }
		out_occluded[i] = trace(s, v3(r), v3(r + 4), r[3], r[7], true, &k, &t, b) ? 1 : 0;
	}
	return 0;
}

// BSDF cases in the layout of pgpu_bsdf_eval: cases [n][19], normals [n][6] -> out [n][16].
int port_bsdf(const float* cases, const float* normals, uint32_t n, float* out)
{
	for(uint32_t i = 0; i < n; ++i)
	{
		const float* c = cases + 19 * i;
		const int type = static_cast<int>(c[0]);
		Material m{type, Rgb{c[1], c[2], c[3]}, 0.001f, 1.0f, 1.5f};
		if(type == 1) { m.alpha = std::max(c[1] * c[1], 0.001f); m.c = Rgb{c[2], c[3], c[4]}; }
		if(type == 2) { m.alpha = std::max(c[1] * c[1], 0.001f); m.ior_outer = c[2]; m.ior_inner = c[3]; }
		Surface x;
		x.ng = v3(normals + 6 * i);
		x.ns = v3(normals + 6 * i + 3);
		make_basis(x);
		const Vec v = v3(c + 10), l = v3(c + 13);
		float* o = out + 16 * i;
		std::fill(o, o + 16, 0.0f);
		Rgb f;
		if(bsdf_eval(m, x, l, v, &f)) { o[0] = 1; o[1] = f.r; o[2] = f.g; o[3] = f.b; }
		const float p = bsdf_pdf(m, x, l, v);
		if(p > 0) { o[4] = 1; o[5] = p; }
		const Sample s = bsdf_sample(m, x, v, c[16], c[17], c[18]);
		if(s.ok)
		{
			o[6] = 1; o[7] = s.l.x; o[8] = s.l.y; o[9] = s.l.z;
			o[10] = s.w.r; o[11] = s.w.g; o[12] = s.w.b; o[13] = s.rel_ior; o[14] = std::abs(dot(x.ns, s.l));
		}
	}
	return 0;
}

// Renders a flat scene (layout of pgpu_scene_create) into FP64 sums [h][w][3].
int port_render(const float* tris, const uint32_t* tri_material, const uint32_t* tri_emitter, uint32_t num_tris,
                const float* materials, uint32_t num_materials, const float* emitters, uint32_t num_emitters,
                const float* camera, uint32_t spp, uint32_t max_bounces, uint32_t estimator, uint32_t threads,
                uint64_t seed, double* out_sums)
{
	Scene s;
	if(!setup_scene(s, camera, tris, tri_material, tri_emitter, num_tris, materials, num_materials, emitters, num_emitters))
	{
		return 1;
	}
	s.estimator = estimator;
	render(s, spp, max_bounces, threads, seed, out_sums);
	return 0;
}

// The same with a sample filter (0 box, 1 gaussian, 2 mn, 3 bh): FP64 sums [h][w][4] = R, G, B, W.
int port_render_filtered(const float* tris, const uint32_t* tri_material, const uint32_t* tri_emitter, uint32_t num_tris,
                         const float* materials, uint32_t num_materials, const float* emitters, uint32_t num_emitters,
                         const float* camera, uint32_t spp, uint32_t max_bounces, uint32_t estimator, uint32_t threads,
                         uint64_t seed, uint32_t filter, double* out_sums)
{
	Scene s;
	if(filter > 3 || !setup_scene(s, camera, tris, tri_material, tri_emitter, num_tris, materials, num_materials, emitters, num_emitters))
	{
		return 1;
	}
	s.estimator = estimator;
	render_filtered(s, spp, max_bounces, threads, seed, static_cast<int>(filter), out_sums);
	return 0;
}

}// extern "C"

#ifdef PH_PORT_MAIN
int main(int argc, char** argv)
{
	if(argc < 5)
	{
		std::fprintf(stderr, "usage: %s <scene.bin> <threads> <max-bounces> <out.rgbf32> [repeats]\n", argv[0]);
		return 2;
	}
	FILE* f = std::fopen(argv[1], "rb");
	if(!f) { return 1; }
	std::vector<unsigned char> buf;
	unsigned char tmp[1 << 16];
	std::size_t got;
	while((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) { buf.insert(buf.end(), tmp, tmp + got); }
	std::fclose(f);
	std::size_t off = 0;
	auto take = [&](std::size_t bytes) { const unsigned char* p = buf.data() + off; off += bytes; return p; };
	if(buf.size() < 8 || std::memcmp(take(4), "PHPT", 4) != 0) { return 1; }
	uint32_t hdr[5];
	std::memcpy(hdr, take(20), 20);
	float cam[12];
	std::memcpy(cam, take(48), 48);
	uint32_t counts[3];
	std::memcpy(counts, take(12), 12);
	const uint32_t n = counts[0], nm = counts[1], ne = counts[2];
	std::vector<float> tris(9 * n), mats(8 * nm), ems(4 * ne);
	std::vector<uint32_t> tm(n), te(n);
	std::memcpy(tris.data(), take(36 * n), 36 * n);
	std::memcpy(tm.data(), take(4 * n), 4 * n);
	std::memcpy(te.data(), take(4 * n), 4 * n);
	std::memcpy(mats.data(), take(32 * nm), 32 * nm);
	if(ne) { std::memcpy(ems.data(), take(16 * ne), 16 * ne); }
	const uint32_t threads = static_cast<uint32_t>(std::atoi(argv[2]));
	const uint32_t bounces = static_cast<uint32_t>(std::atoi(argv[3]));
	const int repeats = argc >= 6 ? std::max(1, std::atoi(argv[5])) : 1;
	using Clock = std::chrono::steady_clock;
	const auto t0 = Clock::now();
	Scene s;
	setup_scene(s, cam, tris.data(), tm.data(), te.data(), n, mats.data(), nm, ems.data(), ne);
	s.estimator = hdr[4];
	const auto t1 = Clock::now();
	std::vector<double> sums(3ull * s.width * s.height);
	for(int rep = 0; rep < repeats; ++rep)
	{
		const auto a = Clock::now();
		render(s, hdr[3], bounces, threads, 42 + rep, sums.data());
		const auto b = Clock::now();
		std::vector<float> img(sums.size());
		for(std::size_t i = 0; i < img.size(); ++i) { img[i] = static_cast<float>(sums[i] / hdr[3]); }
		FILE* o = std::fopen(argv[4], "wb");
		if(o) { std::fwrite(img.data(), 4, img.size(), o); std::fclose(o); }
		std::printf("{\"width\": %u, \"height\": %u, \"threads\": %u, \"max_bounces\": %u, \"repeat\": %d, "
		            "\"load_s\": 0.0, \"update_s\": %.6f, \"render_s\": %.6f}\n",
		            s.width, s.height, threads, bounces, rep,
		            std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(b - a).count());
		std::fflush(stdout);
	}
	return 0;
}
#endif
