// Learned path guiding: network shape, input encoding and the von Mises-Fisher lobe mixture.
//
// The reference renderer has no guiding; this is the learned proposal the GPU estimator adds on
// top of BSDF sampling (combined by one-sample MIS, so the estimator stays unbiased). A small MLP
// maps a surface point to a mixture of 8 vMF lobes over incident directions:
//
//   input   7 scalars in [0, 1]: position (3, scene-bound normalised), shading normal (2, polar
//           angles / pi and 2 pi) and outgoing direction (2, same), each one-blob encoded into 32
//           bins (Mueller et al. 2019, "Neural Importance Sampling"): 224 features;
//   hidden  4 layers of 64 ReLU units;
//   output  8 lobes x (weight logit, mean direction xyz, log concentration) = 40 values.
//
// Weights are BF16 on the tensor cores, accumulation FP32; the master copy and Adam moments are
// FP32. Parameter order in the packed FP32 vector: W0[224][64], b0[64], W1[64][64], b1[64],
// W2[64][64], b2[64], W3[64][64], b3[64], W4[64][40], b4[40] (W[in][out], row-major).
#pragma once

#include "bsdf.cuh"

namespace pg
{
namespace guide
{

constexpr int kInputs = 7;
constexpr int kBins = 32;
constexpr int kIn = kInputs * kBins;      // 224 = 14 MMA K-steps of 16
constexpr int kHidden = 64;
constexpr int kHiddenLayers = 4;
constexpr int kLobes = 8;
constexpr int kOut = kLobes * 5;          // 40
constexpr int kOutPad = 48;               // MMA N must be a multiple of 16 at M = 128
constexpr int kTile = 128;                // rows per tcgen05 tile (MMA M)
// Decoded mixture row written for the renderer: per lobe (weight, mean xyz, kappa, weight x vMF
// normalisation), so that the density is sum_j c_j exp(kappa_j (mu_j . w - 1)).
constexpr int kMixFloats = kLobes * 6;

constexpr int kOffW0 = 0;
constexpr int kOffB0 = kOffW0 + kIn * kHidden;
constexpr int kOffW1 = kOffB0 + kHidden;
constexpr int kOffB1 = kOffW1 + kHidden * kHidden;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kHidden * kHidden;
constexpr int kOffW4 = kOffB3 + kHidden;
constexpr int kOffB4 = kOffW4 + kHidden * kOut;
constexpr int kNumParams = kOffB4 + kOut;  // 29,480

constexpr float kMinKappa = 1e-2f;
constexpr float kMaxKappa = 5e3f;

// One-blob encoding: a Gaussian of width 1/kBins centred on the input, sampled at bin centres.
PG_HD float one_blob(float s, int bin)
{
	const float c = (static_cast<float>(bin) + 0.5f) / kBins;
	const float z = (s - c) * kBins;
	return expf(-0.5f * z * z);
}

// Query features: 7 scalars in [0, 1].
struct Features
{
	float v[kInputs];
};

PG_HD float wrap01(float x)
{
	return fminf(fmaxf(x, 0.0f), 1.0f);
}

// Direction -> (theta / pi, (phi + pi) / (2 pi)), theta from +z.
PG_HD void dir_to_unit2(V3 d, float* a, float* b)
{
	const float theta = acosf(fminf(fmaxf(d.z, -1.0f), 1.0f));
	const float phi = atan2f(d.y, d.x);
	*a = wrap01(theta * (1.0f / kPi));
	*b = wrap01((phi + kPi) * (0.5f / kPi));
}

PG_HD Features make_features(V3 pos, V3 scene_lo, V3 scene_extent_rcp, V3 normal, V3 wo)
{
	Features f;
	f.v[0] = wrap01((pos.x - scene_lo.x) * scene_extent_rcp.x);
	f.v[1] = wrap01((pos.y - scene_lo.y) * scene_extent_rcp.y);
	f.v[2] = wrap01((pos.z - scene_lo.z) * scene_extent_rcp.z);
	dir_to_unit2(normal, &f.v[3], &f.v[4]);
	dir_to_unit2(wo, &f.v[5], &f.v[6]);
	return f;
}

// Decoded mixture: weights sum to one, unit means, concentrations in [kMinKappa, kMaxKappa].
struct Mixture
{
	float w[kLobes];
	V3    mu[kLobes];
	float kappa[kLobes];
};

// Raw network outputs (40) -> mixture. Softmax over logits; mean = raw xyz normalised (falls back
// to +z for a zero vector); kappa = exp(raw) clamped.
PG_HD Mixture decode(const float* raw)
{
	Mixture m;
	float mx = -3.0e38f;
	for(int j = 0; j < kLobes; ++j)
	{
		mx = fmaxf(mx, raw[5 * j]);
	}
	float sum = 0.0f;
	for(int j = 0; j < kLobes; ++j)
	{
		m.w[j] = expf(raw[5 * j] - mx);
		sum += m.w[j];
	}
	for(int j = 0; j < kLobes; ++j)
	{
		m.w[j] /= sum;
		V3 d = v3(raw[5 * j + 1], raw[5 * j + 2], raw[5 * j + 3]);
		const float l2 = dot(d, d);
		m.mu[j] = l2 > 1e-20f ? d * (1.0f / sqrtf(l2)) : v3(0.0f, 0.0f, 1.0f);
		m.kappa[j] = fminf(fmaxf(expf(raw[5 * j + 4]), kMinKappa), kMaxKappa);
	}
	return m;
}

// vMF density on the unit sphere: kappa / (2 pi (1 - exp(-2 kappa))) exp(kappa (mu.w - 1)).
PG_HD float vmf_pdf(V3 mu, float kappa, V3 w)
{
	const float norm = kappa / (2.0f * kPi * (1.0f - expf(-2.0f * kappa)));
	return norm * expf(kappa * (dot(mu, w) - 1.0f));
}

PG_HD float mixture_pdf(const Mixture& m, V3 w)
{
	float p = 0.0f;
	for(int j = 0; j < kLobes; ++j)
	{
		p += m.w[j] * vmf_pdf(m.mu[j], m.kappa[j], w);
	}
	return p;
}

// A direction from one vMF lobe (mean n, concentration k) by (u1, u2) (W. Jakob, "Numerically
// stable sampling of the von Mises Fisher distribution on S2", 2012).
PG_HD V3 vmf_sample(V3 n, float k, float u1, float u2)
{
	const float w = 1.0f + logf(fmaxf(u1 + (1.0f - u1) * expf(-2.0f * k), 1e-30f)) / k;
	const float s = sqrtf(fmaxf(0.0f, 1.0f - w * w));
	const float phi = 2.0f * kPi * u2;
	const V3 local = v3(s * cosf(phi), s * sinf(phi), w);
	// orthonormal basis around mu (Duff et al. 2017)
	const float sign = n.z >= 0.0f ? 1.0f : -1.0f;
	const float a = -1.0f / (sign + n.z);
	const float b = n.x * n.y * a;
	const V3 t = v3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
	const V3 bt = v3(b, sign + n.y * n.y * a, -n.y);
	return normalize(t * local.x + bt * local.y + n * local.z);
}

// Samples one lobe by u0, then a direction from it by (u1, u2).
PG_HD V3 mixture_sample(const Mixture& m, float u0, float u1, float u2)
{
	int j = 0;
	float acc = m.w[0];
	while(j < kLobes - 1 && u0 >= acc)
	{
		++j;
		acc += m.w[j];
	}
	return vmf_sample(m.mu[j], m.kappa[j], u1, u2);
}

}// end namespace guide
}// end namespace pg
