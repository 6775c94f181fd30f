// Golden-vector extractor over the reference's own classes (test infrastructure only).
//
// hits  <tris.f32> <rays.f32> <out.bin>
//     Builds PTriangle primitives (Engine/Source/Core/Intersection/PTriangle.cpp:19-35) from the
//     given vertices, a TBinaryBvhIntersector<size_t> over them (the reference's default TLAS,
//     Engine/Source/Core/Intersection/BVH/TBinaryBvhIntersector.ipp:20-97), and answers each
//     ray with isIntersecting (closest primitive index, t, barycentrics) and isOccluding.
//     tris: float32 [N][3][3]; rays: float32 [M][8] = origin(3), minT, direction(3), maxT.
//     out:  per ray int32 prim (-1 = miss), float32 t, b0, b1, b2, int32 occluded.
//
// energy <r> <g> <b> <watts>   (see run_energy)
//
// lights <groups.f32> <queries.f32> <out.f32>
//     Light selection and direct-light densities of the reference's power-favouring emitter
//     sampler (Engine/Source/Core/Emitter/Sampler/ESPowerFavoring.cpp:21-97) over area emitters
//     made as AAreaLight makes them (Engine/Source/Actor/Light/AAreaLight.cpp:72-85): one
//     DiffuseSurfaceEmitter for a single triangle, else a GroupedDiffuseSurfaceEmitter, each with a
//     constant radiance texture.
//     groups (float32): G, then per group: n, r, g, b, n x 9 vertex coordinates.
//     queries (float32 x 6 per query): target position (3), group, triangle within the group,
//        pad; the light point is the triangle's centroid seen along the ray target -> centroid.
//     out (float32): per group: flux weight (Emitter::calcRadiantFluxApprox, the weight
//        ESPowerFavoring::update gives it) and pick probability (the sampler's own distribution,
//        TPwcDistribution1D::pdfDiscrete); then per query: pdfW of ESPowerFavoring::calcDirectPdf
//        (0 where no pdf), pdfW of the emitter alone (without the pick), 1 if the ray towards the
//        centroid hit the triangle (else 0 and no densities), and the emission point that hit
//        produced (3).
//
// bsdf  <cases.f32> <out.f32>
//     Evaluates LambertianReflector, OpaqueMicrofacet (IsoTrowbridgeReitzConstant + Schlick) and
//     TranslucentMicrofacet (IsoTrowbridgeReitzConstant + exact dielectric Fresnel) through the
//     SurfaceOptics entry points used by the estimators (calcBsdf / calcBsdfPdf / genBsdfSample,
//     Engine/Source/Core/SurfaceBehavior/SurfaceOptics.cpp) with the Strict sidedness context,
//     at a surface point of a large triangle whose face normal is the case's N.
//     case (float32 x 19): type, p0..p5, N(3), V(3), L(3), u(3)
//        type 0 Lambertian: p0..p2 albedo
//        type 1 conductor:  p0 roughness, p1..p3 f0
//        type 2 dielectric: p0 roughness, p1 ior outer, p2 ior inner
//     out (float32 x 22): eval_ok, bsdf(3), pdf_ok, pdfW, sample_ok, L(3), pdfAppliedBsdfCos(3),
//        relativeIor, sample_cos, pad, Ng(3), Ns(3) -- the last two are the surface normals the
//        reference derived from the triangle, which the GPU side must use to compare like for like
#include "Core/Intersection/PTriangle.h"
#include "Core/Intersection/PrimitiveMetadata.h"
#include "Core/Emitter/DiffuseSurfaceEmitter.h"
#include "Core/Emitter/GroupedDiffuseSurfaceEmitter.h"
#include "Core/Emitter/Sampler/ESPowerFavoring.h"
#include "Core/Emitter/Query/DirectEnergyPdfQuery.h"
#include "Math/Random/TPwcDistribution1D.h"
#include "Core/Intersection/BVH/TBinaryBvhIntersector.h"
#include "Core/HitProbe.h"
#include "Core/Ray.h"
#include "Core/SurfaceHit.h"
#include "Core/SurfaceBehavior/SurfaceOptics/LambertianReflector.h"
#include "Core/SurfaceBehavior/SurfaceOptics/OpaqueMicrofacet.h"
#include "Core/SurfaceBehavior/SurfaceOptics/TranslucentMicrofacet.h"
#include "Core/SurfaceBehavior/Property/IsoTrowbridgeReitzConstant.h"
#include "Core/SurfaceBehavior/Property/SchlickApproxConductorFresnel.h"
#include "Core/SurfaceBehavior/Property/ExactDielectricFresnel.h"
#include "Core/SurfaceBehavior/BsdfQueryContext.h"
#include "Core/SurfaceBehavior/BsdfEvalQuery.h"
#include "Core/SurfaceBehavior/BsdfSampleQuery.h"
#include "Core/SurfaceBehavior/BsdfPdfQuery.h"
#include "Core/SampleGenerator/SampleFlow.h"
#include "Core/Texture/constant_textures.h"
#include "Math/TVector3.h"
#include "Math/Color/Spectrum.h"
#include "Utility/TSpan.h"

#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

using namespace ph;

namespace
{

std::vector<float> read_f32(const char* path)
{
	std::vector<float> v;
	FILE* f = std::fopen(path, "rb");
	if(!f)
	{
		return v;
	}
	std::fseek(f, 0, SEEK_END);
	const long n = std::ftell(f);
	std::fseek(f, 0, SEEK_SET);
	v.resize(static_cast<std::size_t>(n) / sizeof(float));
	if(std::fread(v.data(), sizeof(float), v.size(), f) != v.size())
	{
		v.clear();
	}
	std::fclose(f);
	return v;
}

int run_hits(const char* trisPath, const char* raysPath, const char* outPath)
{
	const auto tris = read_f32(trisPath);
	const auto rays = read_f32(raysPath);
	if(tris.empty() || tris.size() % 9 != 0 || rays.size() % 8 != 0)
	{
		std::fprintf(stderr, "bad inputs\n");
		return 1;
	}
	const std::size_t numTris = tris.size() / 9;
	const std::size_t numRays = rays.size() / 8;

	std::vector<std::unique_ptr<PTriangle>> prims;
	std::vector<const Intersectable*> items;
	std::unordered_map<const Intersectable*, int32_t> indexOf;
	prims.reserve(numTris);
	for(std::size_t i = 0; i < numTris; ++i)
	{
		const float* v = &tris[9 * i];
		prims.push_back(std::make_unique<PTriangle>(
			math::Vector3R(v[0], v[1], v[2]),
			math::Vector3R(v[3], v[4], v[5]),
			math::Vector3R(v[6], v[7], v[8])));
		items.push_back(prims.back().get());
		indexOf[prims.back().get()] = static_cast<int32_t>(i);
	}

	TBinaryBvhIntersector<std::size_t> bvh;
	bvh.update(TSpanView<const Intersectable*>(items.data(), items.size()));

	FILE* out = std::fopen(outPath, "wb");
	if(!out)
	{
		return 1;
	}
	for(std::size_t r = 0; r < numRays; ++r)
	{
		const float* q = &rays[8 * r];
		const Ray ray(
			math::Vector3R(q[0], q[1], q[2]),
			math::Vector3R(q[4], q[5], q[6]),
			q[3], q[7]);

		HitProbe probe;
		int32_t prim = -1;
		float t = 0.0f, b[3] = {0.0f, 0.0f, 0.0f};
		if(bvh.isIntersecting(ray, probe))
		{
			const auto it = indexOf.find(probe.getTopHit());
			prim = it == indexOf.end() ? -2 : it->second;
			t = probe.getHitRayT();
			HitProbe copy = probe;
			const auto bary = copy.popCache<math::Vector3R>();
			b[0] = bary.x(); b[1] = bary.y(); b[2] = bary.z();
		}
		const int32_t occluded = bvh.isOccluding(ray) ? 1 : 0;
		std::fwrite(&prim, 4, 1, out);
		std::fwrite(&t, 4, 1, out);
		std::fwrite(b, 4, 3, out);
		std::fwrite(&occluded, 4, 1, out);
	}
	std::fclose(out);
	return 0;
}

int run_bsdf(const char* casesPath, const char* outPath)
{
	const auto cases = read_f32(casesPath);
	constexpr std::size_t kIn = 19;
	constexpr std::size_t kOut = 22;
	if(cases.empty() || cases.size() % kIn != 0)
	{
		std::fprintf(stderr, "bad cases\n");
		return 1;
	}
	const std::size_t n = cases.size() / kIn;
	std::vector<float> out(n * kOut, 0.0f);

	for(std::size_t i = 0; i < n; ++i)
	{
		const float* c = &cases[kIn * i];
		const int type = static_cast<int>(c[0]);
		const math::Vector3R N(c[7], c[8], c[9]);
		const math::Vector3R V(c[10], c[11], c[12]);
		const math::Vector3R L(c[13], c[14], c[15]);
		const real u[3] = {c[16], c[17], c[18]};

		std::unique_ptr<SurfaceOptics> optics;
		if(type == 0)
		{
			optics = std::make_unique<LambertianReflector>(
				std::make_shared<TConstantTexture<math::Spectrum>>(math::Spectrum(std::array<real, 3>{c[1], c[2], c[3]})));
		}
		else if(type == 1)
		{
			optics = std::make_unique<OpaqueMicrofacet>(
				std::make_shared<SchlickApproxConductorFresnel>(math::Spectrum(std::array<real, 3>{c[2], c[3], c[4]})),
				std::make_shared<IsoTrowbridgeReitzConstant>(c[1] * c[1], EMaskingShadowing::HightCorrelated));
		}
		else
		{
			optics = std::make_unique<TranslucentMicrofacet>(
				std::make_shared<ExactDielectricFresnel>(c[2], c[3]),
				std::make_shared<IsoTrowbridgeReitzConstant>(c[1] * c[1], EMaskingShadowing::HightCorrelated));
		}

		// A large triangle through the origin with face normal N; the surface point is where a
		// ray along -N from N hits it.
		const math::Vector3R helper = std::abs(N.y()) < 0.9f ? math::Vector3R(0, 1, 0) : math::Vector3R(1, 0, 0);
		const math::Vector3R T = helper.cross(N).normalize();
		const math::Vector3R B = N.cross(T).normalize();
		math::Vector3R va = T.mul(-10.0_r).add(B.mul(-10.0_r));
		math::Vector3R vb = T.mul(10.0_r).add(B.mul(-10.0_r));
		math::Vector3R vc = B.mul(10.0_r);
		if((vb - va).cross(vc - va).dot(N) < 0)
		{
			std::swap(vb, vc);
		}
		PTriangle tri(va, vb, vc);
		const Ray ray(N.mul(0.5_r), N.mul(-1.0_r), 0, 10);
		HitProbe probe;
		if(!tri.isIntersecting(ray, probe))
		{
			std::fprintf(stderr, "case %zu: constructed surface not hit\n", i);
			return 1;
		}
		const SurfaceHit X(ray, probe, SurfaceHitReason(ESurfaceHitReason::IncidentRay));
		float* o = &out[kOut * i];

		{
			const auto ng = X.getGeometryNormal();
			const auto ns = X.getShadingNormal();
			o[16] = ng.x(); o[17] = ng.y(); o[18] = ng.z();
			o[19] = ns.x(); o[20] = ns.y(); o[21] = ns.z();
		}

		BsdfQueryContext ctx(lta::ESidednessPolicy::Strict);
		{
			BsdfEvalQuery eval(ctx);
			eval.inputs.set(X, L, V);
			optics->calcBsdf(eval);
			if(eval.outputs.isMeasurable())
			{
				const auto f = eval.outputs.getBsdf();
				o[0] = 1.0f; o[1] = f[0]; o[2] = f[1]; o[3] = f[2];
			}
		}
		{
			BsdfPdfQuery pdf(ctx);
			BsdfEvalQuery evalInputs(ctx);
			evalInputs.inputs.set(X, L, V);
			pdf.inputs.set(evalInputs.inputs);
			optics->calcBsdfPdf(pdf);
			if(pdf.outputs)
			{
				o[4] = 1.0f;
				o[5] = pdf.outputs.getSampleDirPdfW();
			}
		}
		{
			BsdfSampleQuery sample(ctx);
			sample.inputs.set(X, V);
			SampleFlow flow(u, 3);
			optics->genBsdfSample(sample, flow);
			if(sample.outputs.isMeasurable())
			{
				const auto Ls = sample.outputs.getL();
				const auto w = sample.outputs.getPdfAppliedBsdfCos();
				o[6] = 1.0f;
				o[7] = Ls.x(); o[8] = Ls.y(); o[9] = Ls.z();
				o[10] = w[0]; o[11] = w[1]; o[12] = w[2];
				o[13] = sample.outputs.getRelativeIor();
				o[14] = sample.outputs.getCos();
			}
		}
	}

	FILE* f = std::fopen(outPath, "wb");
	if(!f)
	{
		return 1;
	}
	std::fwrite(out.data(), sizeof(float), out.size(), f);
	std::fclose(f);
	return 0;
}

// A triangle carrying the metadata that ties it to its emitter, as cooked light primitives do
// (ESPowerFavoring::calcDirectPdf finds the emitter through the hit primitive's metadata).
class EmitterTriangle : public PTriangle
{
public:
	EmitterTriangle(const math::Vector3R& a, const math::Vector3R& b, const math::Vector3R& c,
	                const PrimitiveMetadata* metadata)
		: PTriangle(a, b, c), m_metadata(metadata)
	{}

	const PrimitiveMetadata* getMetadata() const override { return m_metadata; }

private:
	const PrimitiveMetadata* m_metadata;
};

int run_lights(const char* groupsPath, const char* queriesPath, const char* outPath)
{
	const auto g = read_f32(groupsPath);
	const auto q = read_f32(queriesPath);
	if(g.empty() || q.size() % 6 != 0)
	{
		std::fprintf(stderr, "bad inputs\n");
		return 1;
	}
	const std::size_t numGroups = static_cast<std::size_t>(g[0]);
	std::vector<std::unique_ptr<PrimitiveMetadata>> metas;
	std::vector<std::vector<std::unique_ptr<EmitterTriangle>>> tris(numGroups);
	std::vector<std::vector<math::Vector3R>> centroids(numGroups);
	std::vector<std::unique_ptr<Emitter>> emitters;
	std::vector<const Emitter*> emitterPtrs;
	std::size_t at = 1;
	for(std::size_t k = 0; k < numGroups; ++k)
	{
		const std::size_t n = static_cast<std::size_t>(g.at(at));
		const math::Spectrum radiance(std::array<real, 3>{g.at(at + 1), g.at(at + 2), g.at(at + 3)});
		at += 4;
		metas.push_back(std::make_unique<PrimitiveMetadata>());
		std::vector<const Primitive*> prims;
		for(std::size_t i = 0; i < n; ++i, at += 9)
		{
			const math::Vector3R va(g.at(at + 0), g.at(at + 1), g.at(at + 2));
			const math::Vector3R vb(g.at(at + 3), g.at(at + 4), g.at(at + 5));
			const math::Vector3R vc(g.at(at + 6), g.at(at + 7), g.at(at + 8));
			tris[k].push_back(std::make_unique<EmitterTriangle>(va, vb, vc, metas.back().get()));
			centroids[k].push_back(va.add(vb).add(vc).div(3.0_r));
			prims.push_back(tris[k].back().get());
		}
		auto texture = std::make_shared<TConstantTexture<math::Spectrum>>(radiance);
		if(prims.size() == 1)
		{
			emitters.push_back(std::make_unique<DiffuseSurfaceEmitter>(prims[0], texture));
		}
		else
		{
			emitters.push_back(std::make_unique<GroupedDiffuseSurfaceEmitter>(
				TSpanView<const Primitive*>(prims.data(), prims.size()), texture));
		}
		metas.back()->getSurface().setEmitter(emitters.back().get());
		emitterPtrs.push_back(emitters.back().get());
	}

	ESPowerFavoring sampler;
	sampler.update(TSpanView<const Emitter*>(emitterPtrs.data(), emitterPtrs.size()));

	// the same weights and distribution ESPowerFavoring::update builds (ESPowerFavoring.cpp:41-49)
	std::vector<real> weights(numGroups);
	for(std::size_t k = 0; k < numGroups; ++k)
	{
		weights[k] = emitterPtrs[k]->calcRadiantFluxApprox();
	}
	const math::TPwcDistribution1D<real> distribution(weights);

	std::vector<float> out;
	for(std::size_t k = 0; k < numGroups; ++k)
	{
		out.push_back(weights[k]);
		out.push_back(distribution.pdfDiscrete(k));
	}
	for(std::size_t i = 0; i < q.size() / 6; ++i)
	{
		const float* r = &q[6 * i];
		const math::Vector3R target(r[0], r[1], r[2]);
		const auto& tri = *tris.at(static_cast<std::size_t>(r[3])).at(static_cast<std::size_t>(r[4]));
		const math::Vector3R centroid = centroids.at(static_cast<std::size_t>(r[3])).at(static_cast<std::size_t>(r[4]));
		const math::Vector3R dir = centroid.sub(target);
		const Ray ray(target, dir.normalize(), 0, dir.length() * 2.0_r);
		HitProbe probe;
		float pdfW = 0.0f, emitterPdfW = 0.0f, hit = 0.0f, pos[3] = {0.0f, 0.0f, 0.0f};
		if(tri.isIntersecting(ray, probe))
		{
			hit = 1.0f;
			const SurfaceHit Xe(ray, probe, SurfaceHitReason(ESurfaceHitReason::IncidentRay));
			pos[0] = Xe.getPos().x(); pos[1] = Xe.getPos().y(); pos[2] = Xe.getPos().z();
			DirectEnergyPdfQuery query;
			query.inputs.set(target, Xe);
			sampler.calcDirectPdf(query);
			if(query.outputs)
			{
				pdfW = query.outputs.getPdfW();
			}
			DirectEnergyPdfQuery alone;
			alone.inputs.set(target, Xe);
			emitterPtrs.at(static_cast<std::size_t>(r[3]))->calcDirectPdf(alone);
			if(alone.outputs)
			{
				emitterPdfW = alone.outputs.getPdfW();
			}
		}
		out.push_back(pdfW);
		out.push_back(emitterPdfW);
		out.push_back(hit);
		out.push_back(pos[0]);
		out.push_back(pos[1]);
		out.push_back(pos[2]);
	}

	FILE* f = std::fopen(outPath, "wb");
	if(!f)
	{
		return 1;
	}
	std::fwrite(out.data(), sizeof(float), out.size(), f);
	std::fclose(f);
	return 0;
}

}// end anonymous namespace

// energy <r> <g> <b> <watts>: the radiance colour an area light of that colour and power gets,
// Spectrum(color).putEnergy(watts) (Engine/Source/Actor/Light/AAreaLight.cpp:57-58), and the
// relative luminance of the colour.
int run_energy(float r, float g, float b, float watts)
{
	const math::Spectrum c(std::array<real, 3>{r, g, b});
	const auto e = math::Spectrum(c).putEnergy(watts);
	std::printf("%.9g %.9g %.9g %.9g\n", e[0], e[1], e[2], c.relativeLuminance());
	return 0;
}

int main(int argc, char** argv)
{
	if(argc >= 6 && std::string(argv[1]) == "energy")
	{
		return run_energy(std::stof(argv[2]), std::stof(argv[3]), std::stof(argv[4]), std::stof(argv[5]));
	}
	if(argc >= 5 && std::string(argv[1]) == "hits")
	{
		return run_hits(argv[2], argv[3], argv[4]);
	}
	if(argc >= 4 && std::string(argv[1]) == "bsdf")
	{
		return run_bsdf(argv[2], argv[3]);
	}
	if(argc >= 5 && std::string(argv[1]) == "lights")
	{
		return run_lights(argv[2], argv[3], argv[4]);
	}
	std::fprintf(stderr, "usage: %s hits <tris> <rays> <out> | bsdf <cases> <out> | lights <groups> <queries> <out>\n", argv[0]);
	return 2;
}
