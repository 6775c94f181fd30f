#include "engine.h"
#include "ply.h"
#include "pg_render_object.h"
#include "scene_build.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace pg
{
namespace
{

constexpr double kPiD = 3.14159265358979323846;

std::string lower(std::string s)
{
	for(char& c : s) { c = static_cast<char>(std::tolower(static_cast<unsigned char>(c))); }
	return s;
}

struct Quat
{
	double w, x, y, z;
};

Quat quat_mul(const Quat& a, const Quat& b)
{
	return Quat{a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
	            a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
	            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
	            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}

void quat_rotate(const double q[4], const double v[3], double out[3])
{
	const Quat p{0.0, v[0], v[1], v[2]};
	const Quat qq{q[0], q[1], q[2], q[3]};
	const Quat qc{q[0], -q[1], -q[2], -q[3]};
	const Quat r = quat_mul(quat_mul(qq, p), qc);
	out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

}// end anonymous namespace

Engine::Engine() = default;
Engine::~Engine() = default;

void Engine::record_error(const std::string& msg)
{
	std::lock_guard<std::mutex> lock(m_error_mutex);
	std::fprintf(stderr, "[photon-gpu] %s\n", msg.c_str());
	if(!m_errors.empty())
	{
		m_errors += "\n";
	}
	m_errors += msg;
}

std::string Engine::last_error() const
{
	std::lock_guard<std::mutex> lock(m_error_mutex);
	return m_errors;
}

void Engine::enter_command(std::string_view fragment)
{
	try
	{
		m_parser.feed(fragment, [this](SdlCommand&& c) { handle(std::move(c)); });
	}
	catch(const std::exception& e)
	{
		record_error(e.what());
	}
}

bool Engine::load_commands(const std::string& path)
{
	std::string full = path;
	if(!path.empty() && path[0] != '/')
	{
		std::ifstream probe(path);
		if(!probe.good())
		{
			full = m_working_dir + "/" + path;
		}
	}
	std::ifstream in(full, std::ios::binary);
	if(!in)
	{
		record_error("cannot open scene file " + full);
		return false;
	}
	std::ostringstream ss;
	ss << in.rdbuf();
	const std::string text = ss.str();
	// A file is a sequence of complete commands; feed in large chunks.
	const std::size_t before = m_parser.num_errors();
	enter_command(text);
	enter_command(";");
	return m_parser.num_errors() == before;
}

void Engine::handle(SdlCommand&& cmd)
{
	if(cmd.kind == SdlCommand::Kind::Directive)
	{
		return;
	}
	if(cmd.kind == SdlCommand::Kind::Load)
	{
		Resource r;
		r.category = cmd.category;
		r.type = cmd.type;
		r.name = cmd.name;
		r.clauses = std::move(cmd.clauses);
		if(r.category == "actor" && m_resources.find(r.name) == m_resources.end())
		{
			m_actor_order.push_back(r.name);
		}
		m_resources[r.name] = std::move(r);
		return;
	}
	// execution: transforms on actors
	auto it = m_resources.find(cmd.name);
	if(it == m_resources.end())
	{
		throw std::runtime_error("execution on unknown resource @" + cmd.name);
	}
	Resource& r = it->second;
	const std::string fn = lower(cmd.function);
	if(fn == "translate")
	{
		const SdlClause* c = cmd.find("amount");
		const auto v = c ? sdl_numbers(c->value) : std::vector<double>{};
		if(v.size() != 3 && v.size() != 1)
		{
			throw std::runtime_error("translate needs a vector3 amount");
		}
		for(int a = 0; a < 3; ++a) { r.pos[a] += v[v.size() == 3 ? a : 0]; }
	}
	else if(fn == "rotate")
	{
		const SdlClause* ca = cmd.find("axis");
		const SdlClause* cd = cmd.find("degrees");
		const SdlClause* cq = cmd.find("rotation");
		Quat add{1, 0, 0, 0};
		if(ca && cd)
		{
			const auto ax = sdl_numbers(ca->value);
			const double deg = sdl_numbers(cd->value).at(0);
			const double len = std::sqrt(ax.at(0) * ax[0] + ax.at(1) * ax[1] + ax.at(2) * ax[2]);
			const double half = deg * kPiD / 180.0 * 0.5;
			const double s = std::sin(half) / len;
			add = Quat{std::cos(half), ax[0] * s, ax[1] * s, ax[2] * s};
		}
		else if(cq)
		{
			const auto q = sdl_numbers(cq->value);
			add = Quat{q.at(3), q.at(0), q.at(1), q.at(2)};
		}
		else
		{
			throw std::runtime_error("rotate needs axis + degrees or a rotation quaternion");
		}
		const Quat cur{r.rot[0], r.rot[1], r.rot[2], r.rot[3]};
		Quat total = quat_mul(add, cur);
		const double n = std::sqrt(total.w * total.w + total.x * total.x + total.y * total.y + total.z * total.z);
		r.rot[0] = total.w / n; r.rot[1] = total.x / n; r.rot[2] = total.y / n; r.rot[3] = total.z / n;
	}
	else if(fn == "scale")
	{
		const SdlClause* c = cmd.find("amount");
		const auto v = c ? sdl_numbers(c->value) : std::vector<double>{};
		if(v.size() != 3 && v.size() != 1)
		{
			throw std::runtime_error("scale needs a vector3 amount");
		}
		for(int a = 0; a < 3; ++a) { r.scale[a] *= v[v.size() == 3 ? a : 0]; }
	}
	else
	{
		throw std::runtime_error("unsupported execution " + cmd.function + "(@" + cmd.name + ")");
	}
}

namespace
{

const SdlClause* find(const std::vector<SdlClause>& cs, const char* name)
{
	for(const auto& c : cs)
	{
		if(c.name == name)
		{
			return &c;
		}
	}
	return nullptr;
}

double get_real(const std::vector<SdlClause>& cs, const char* name, double fallback)
{
	const SdlClause* c = find(cs, name);
	if(!c || c->value.empty())
	{
		return fallback;
	}
	return sdl_numbers(c->value).at(0);
}

bool get_vec3(const std::vector<SdlClause>& cs, const char* name, double out[3])
{
	const SdlClause* c = find(cs, name);
	if(!c)
	{
		return false;
	}
	const auto v = sdl_numbers(c->value);
	if(v.size() == 1)
	{
		out[0] = out[1] = out[2] = v[0];
		return true;
	}
	if(v.size() != 3)
	{
		throw std::runtime_error(std::string("clause ") + name + " needs 3 numbers");
	}
	out[0] = v[0]; out[1] = v[1]; out[2] = v[2];
	return true;
}

double srgb_to_linear(double c)
{
	return c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4);
}

}// end anonymous namespace

void Engine::update()
{
	const auto t0 = std::chrono::steady_clock::now();
	try
	{
		SceneDesc desc;
		cook(desc);
		desc.bvh_builder = m_bvh_builder;
		m_info.num_triangles = desc.tris.size() / 9;
		m_render = make_render_object(std::move(desc));
		m_render->filter = m_filter;
		m_render->scene->set_dome_exact(m_dome_pdf == 1u);
	}
	catch(const std::exception& e)
	{
		m_render.reset();
		record_error(std::string("update failed: ") + e.what());
	}
	m_info.update_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void Engine::cook(SceneDesc& desc)
{
	{
		// ---- session, observer, sample source, visualizer
		const Resource* session = nullptr;
		for(const auto& [name, r] : m_resources)
		{
			if(r.category == "option" && r.type == "single-frame-render-session")
			{
				session = &r;
			}
		}
		if(!session)
		{
			throw std::runtime_error("no single-frame-render-session option in the scene");
		}
		auto ref = [&](const Resource& owner, const char* clause) -> const Resource*
		{
			const SdlClause* c = find(owner.clauses, clause);
			if(!c)
			{
				return nullptr;
			}
			std::string n = c->value;
			if(!n.empty() && n[0] == '@') { n = n.substr(1); }
			auto it = m_resources.find(n);
			return it == m_resources.end() ? nullptr : &it->second;
		};
		uint32_t width = 960, height = 540;
		if(const SdlClause* fs = find(session->clauses, "frame-size"))
		{
			const auto v = sdl_numbers(fs->value);
			if(v.size() != 2)
			{
				throw std::runtime_error("frame-size needs two numbers");
			}
			checked_resolution(v[0], v[1], "frame-size", &width, &height);
		}
		const Resource* observer = ref(*session, "observer");
		const Resource* sampler = ref(*session, "sample-source");
		const Resource* visualizer = ref(*session, "visualizer");
		if(!observer || observer->type != "single-lens")
		{
			throw std::runtime_error("the GPU renderer needs a single-lens observer");
		}
		if(get_real(observer->clauses, "lens-radius-mm", 0.0) > 0.0)
		{
			throw std::runtime_error("thin-lens observers are not supported by the GPU renderer");
		}
		double pos[3] = {0, 0, 0}, dir[3] = {0, 0, -1}, up[3] = {0, 1, 0};
		get_vec3(observer->clauses, "pos", pos);
		get_vec3(observer->clauses, "position", pos);
		const bool has_dir = get_vec3(observer->clauses, "dir", dir) || get_vec3(observer->clauses, "direction", dir);
		const bool has_up = get_vec3(observer->clauses, "up-axis", up);
		if(!has_dir || !has_up)
		{
			double ypr[3] = {0, 0, 0};
			if(get_vec3(observer->clauses, "yaw-pitch-row-degrees", ypr) && (ypr[0] != 0 || ypr[1] != 0 || ypr[2] != 0))
			{
				throw std::runtime_error("yaw-pitch-roll observers are not supported; give dir and up-axis");
			}
		}
		const double sensor_w = get_real(observer->clauses, "sensor-width-mm", 36.0);
		double fov = get_real(observer->clauses, "fov-degrees", -1.0);
		if(fov <= 0.0)
		{
			const double offset = get_real(observer->clauses, "sensor-offset-mm", 36.0);
			fov = 2.0 * std::atan((sensor_w * 0.5) / offset) * 180.0 / kPiD;
		}
		const double samples = sampler ? get_real(sampler->clauses, "samples", 1.0) : 1.0;
		if(!(samples >= 1.0 && samples <= 4294967295.0 && samples == std::floor(samples)))
		{
			throw std::runtime_error("sample-source samples must be a whole number in [1, 2^32 - 1]");
		}
		m_spp = static_cast<uint32_t>(samples);
		m_estimator = PG_EST_BNEEPT;
		m_filter = PG_FILTER_BLACKMAN_HARRIS;
		if(visualizer)
		{
			if(visualizer->type != "path-tracing")
			{
				throw std::runtime_error("visualizer(" + visualizer->type + ") is not the GPU path tracer");
			}
			if(const SdlClause* est = find(visualizer->clauses, "estimator"))
			{
				const std::string e = lower(est->value);
				if(e == "bvpt") { m_estimator = PG_EST_BVPT; }
				else if(e == "bneept") { m_estimator = PG_EST_BNEEPT; }
				else if(e == "bvptdl") { m_estimator = PG_EST_BVPTDL; }
				else { throw std::runtime_error("estimator " + est->value + " is not supported by the GPU renderer"); }
			}
			// sample-filter: box | gaussian | mn | bh, Blackman-Harris when absent
			// (sdl_sample_filter_type.h:18-38, PathTracingVisualizer.h:59-61)
			if(const SdlClause* f = find(visualizer->clauses, "sample-filter"))
			{
				const std::string v = lower(f->value);
				if(v == "box") { m_filter = PG_FILTER_BOX; }
				else if(v == "gaussian") { m_filter = PG_FILTER_GAUSSIAN; }
				else if(v == "mn") { m_filter = PG_FILTER_MITCHELL_NETRAVALI; }
				else if(v == "bh" || v.empty()) { m_filter = PG_FILTER_BLACKMAN_HARRIS; }
				else { throw std::runtime_error("unknown sample-filter " + f->value); }
			}
		}

		// ---- images, materials
		auto image_rgb = [&](const SdlClause& c, double out[3]) -> bool
		{
			if(c.is_reference)
			{
				auto it = m_resources.find(c.value);
				if(it == m_resources.end() || it->second.category != "image" || it->second.type != "constant")
				{
					throw std::runtime_error("only constant images are supported (@" + c.value + ")");
				}
				const auto& ic = it->second.clauses;
				const SdlClause* vals = find(ic, "values");
				if(!vals)
				{
					throw std::runtime_error("constant image without values");
				}
				const auto v = sdl_numbers(vals->value);
				if(v.size() == 1) { out[0] = out[1] = out[2] = v[0]; }
				else if(v.size() == 3) { out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; }
				else { throw std::runtime_error("constant image needs 1 or 3 values"); }
				const SdlClause* cs = find(ic, "color-space");
				if(cs && (lower(cs->value) == "srgb"))
				{
					for(int a = 0; a < 3; ++a) { out[a] = srgb_to_linear(out[a]); }
				}
				return true;
			}
			const auto v = sdl_numbers(c.value);
			if(v.size() == 1) { out[0] = out[1] = out[2] = v[0]; }
			else if(v.size() == 3) { out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; }
			else { throw std::runtime_error("colour needs 1 or 3 numbers"); }
			return true;
		};
		std::map<std::string, uint32_t> material_index;
		desc = SceneDesc{};
		auto material_of = [&](const std::string& name) -> uint32_t
		{
			auto found = material_index.find(name);
			if(found != material_index.end())
			{
				return found->second;
			}
			auto it = m_resources.find(name);
			if(it == m_resources.end() || it->second.category != "material")
			{
				throw std::runtime_error("unknown material @" + name);
			}
			const Resource& m = it->second;
			Material mat{};
			if(m.type == "matte-opaque")
			{
				double a[3] = {0.5, 0.5, 0.5};
				if(const SdlClause* al = find(m.clauses, "albedo")) { image_rgb(*al, a); }
				if(find(m.clauses, "sigma-degrees"))
				{
					throw std::runtime_error("Oren-Nayar (sigma-degrees) is not supported by the GPU renderer");
				}
				mat = make_matte(static_cast<float>(a[0]), static_cast<float>(a[1]), static_cast<float>(a[2]));
			}
			else if(m.type == "abraded-opaque" || m.type == "abraded-translucent")
			{
				const SdlClause* ms = find(m.clauses, "microsurface");
				if(ms && lower(ms->value) != "ggx" && lower(ms->value) != "trowbridge-reitz" && lower(ms->value) != "unspecified")
				{
					throw std::runtime_error("microsurface " + ms->value + " is not supported (GGX only)");
				}
				if(find(m.clauses, "roughness-v"))
				{
					throw std::runtime_error("anisotropic roughness is not supported (isotropic GGX only)");
				}
				const SdlClause* r2a = find(m.clauses, "roughness-to-alpha");
				if(r2a && lower(r2a->value) != "squared")
				{
					throw std::runtime_error("roughness-to-alpha " + r2a->value + " is not supported");
				}
				const SdlClause* msk = find(m.clauses, "masking-shadowing");
				if(msk && lower(msk->value) != "height-correlated")
				{
					throw std::runtime_error("masking-shadowing " + msk->value + " is not supported");
				}
				const double rough = get_real(m.clauses, "roughness", 0.5);
				if(m.type == "abraded-opaque")
				{
					const SdlClause* fr = find(m.clauses, "fresnel");
					if((fr && lower(fr->value) == "exact") || find(m.clauses, "ior-inner-n"))
					{
						throw std::runtime_error("exact conductor Fresnel is not supported (Schlick F0 only)");
					}
					double f0[3] = {1, 1, 1};
					get_vec3(m.clauses, "f0", f0);
					mat = make_conductor(static_cast<float>(rough), static_cast<float>(f0[0]),
					                     static_cast<float>(f0[1]), static_cast<float>(f0[2]));
				}
				else
				{
					const SdlClause* fr = find(m.clauses, "fresnel");
					if(fr && lower(fr->value) != "exact")
					{
						throw std::runtime_error("dielectric Fresnel " + fr->value + " is not supported (exact only)");
					}
					mat = make_dielectric(static_cast<float>(rough),
					                      static_cast<float>(get_real(m.clauses, "ior-outer", 1.0)),
					                      static_cast<float>(get_real(m.clauses, "ior-inner", 1.5)));
				}
			}
			else
			{
				throw std::runtime_error("material(" + m.type + ") is not supported by the GPU renderer");
			}
			desc.materials.push_back(mat);
			const uint32_t idx = static_cast<uint32_t>(desc.materials.size() - 1);
			material_index[name] = idx;
			return idx;
		};
		auto absorber_index = [&]() -> uint32_t
		{
			auto found = material_index.find("@@absorber");
			if(found != material_index.end())
			{
				return found->second;
			}
			Material m{};
			m.type = PG_MAT_ABSORBER;
			desc.materials.push_back(m);
			material_index["@@absorber"] = static_cast<uint32_t>(desc.materials.size() - 1);
			return material_index["@@absorber"];
		};
		auto default_matte_index = [&]() -> uint32_t
		{
			auto found = material_index.find("@@matte");
			if(found != material_index.end())
			{
				return found->second;
			}
			desc.materials.push_back(make_matte(0.5f, 0.5f, 0.5f));
			material_index["@@matte"] = static_cast<uint32_t>(desc.materials.size() - 1);
			return material_index["@@matte"];
		};

		// ---- geometry in local space
		auto geometry_tris = [&](const Resource& g, std::vector<double>& out)
		{
			if(g.type == "triangle-mesh")
			{
				const SdlClause* p = find(g.clauses, "positions");
				const SdlClause* t = find(g.clauses, "texture-coordinates");
				const SdlClause* n = find(g.clauses, "normals");
				if(!p)
				{
					throw std::runtime_error("triangle mesh without positions");
				}
				const auto pos_f = sdl_vector3_array(p->value);
				if(pos_f.empty() || (pos_f.size() / 3) % 3 != 0)
				{
					throw std::runtime_error("triangle mesh with bad/zero position buffer size");
				}
				const std::size_t nv = pos_f.size() / 3;
				if(!t || sdl_vector3_array(t->value).size() / 3 != nv)
				{
					throw std::runtime_error("triangle mesh with mismatched texture-coordinate buffer size");
				}
				if(!n)
				{
					throw std::runtime_error("triangle mesh with mismatched normal buffer size");
				}
				const auto nrm = sdl_vector3_array(n->value);
				if(nrm.size() / 3 != nv)
				{
					throw std::runtime_error("triangle mesh with mismatched normal buffer size");
				}
				for(std::size_t k = 0; k < nrm.size(); ++k)
				{
					if(nrm[k] != 0.0f)
					{
						record_error("vertex normals are ignored: the GPU renderer shades with face normals");
						break;
					}
				}
				out.assign(pos_f.begin(), pos_f.end());
			}
			else if(g.type == "ply")
			{
				const SdlClause* f = find(g.clauses, "ply-file");
				if(!f)
				{
					throw std::runtime_error("ply geometry without ply-file");
				}
				PlyMesh mesh = read_ply(resolve_resource(f->value));
				if(mesh.has_normals)
				{
					record_error("vertex normals are ignored: the GPU renderer shades with face normals");
				}
				if(mesh.tris.empty())
				{
					throw std::runtime_error("ply geometry without faces");
				}
				out = std::move(mesh.tris);
			}
			else if(g.type == "rectangle")
			{
				// GRectangle::genTriangleMesh (Engine/Source/Actor/Geometry/GRectangle.cpp:70-100)
				const double hw = get_real(g.clauses, "width", 1.0) * 0.5;
				const double hh = get_real(g.clauses, "height", 1.0) * 0.5;
				const double A[3] = {-hw, hh, 0}, B[3] = {-hw, -hh, 0}, C[3] = {hw, -hh, 0}, D[3] = {hw, hh, 0};
				const double* tri[6] = {A, B, D, B, C, D};
				out.clear();
				for(const double* v : tri) { out.insert(out.end(), v, v + 3); }
			}
			else
			{
				throw std::runtime_error("geometry(" + g.type + ") is not supported by the GPU renderer");
			}
		};
		auto bake = [](const Resource& actor, const std::vector<double>& local, std::vector<float>& world,
		               bool keep_scale)
		{
			(void)keep_scale;
			const std::size_t nv = local.size() / 3;
			for(std::size_t i = 0; i < nv; ++i)
			{
				double v[3] = {local[3 * i] * actor.scale[0], local[3 * i + 1] * actor.scale[1], local[3 * i + 2] * actor.scale[2]};
				double r[3];
				quat_rotate(actor.rot, v, r);
				world.push_back(static_cast<float>(r[0] + actor.pos[0]));
				world.push_back(static_cast<float>(r[1] + actor.pos[1]));
				world.push_back(static_cast<float>(r[2] + actor.pos[2]));
			}
		};
		auto is_degenerate = [](const float* v)
		{
			const double ax = v[3] - v[0], ay = v[4] - v[1], az = v[5] - v[2];
			const double bx = v[6] - v[0], by = v[7] - v[1], bz = v[8] - v[2];
			const float cx = static_cast<float>(ay * bz - az * by), cy = static_cast<float>(az * bx - ax * bz);
			const float cz = static_cast<float>(ax * by - ay * bx);
			const float l2 = cx * cx + cy * cy + cz * cz;
			return !(l2 > 0.0f) || std::isinf(l2);
		};
		auto add_triangles = [&](const std::vector<float>& world, uint32_t mat, uint32_t emitter_plus_one) -> double
		{
			double area = 0.0;
			for(std::size_t i = 0; i + 9 <= world.size(); i += 9)
			{
				const float* v = &world[i];
				if(is_degenerate(v))
				{
					continue;
				}
				desc.tris.insert(desc.tris.end(), v, v + 9);
				desc.tri_material.push_back(mat);
				desc.tri_emitter.push_back(emitter_plus_one);
				const double ax = v[3] - v[0], ay = v[4] - v[1], az = v[5] - v[2];
				const double bx = v[6] - v[0], by = v[7] - v[1], bz = v[8] - v[2];
				const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
				area += 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
			}
			return area;
		};

		double dome_center[3] = {0, 0, 0};
		bool has_dome = false;
		for(const auto& actor_name : m_actor_order)
		{
			const Resource& a = m_resources.at(actor_name);
			if(a.type == "model")
			{
				const Resource* g = ref(a, "geometry");
				const SdlClause* mc = find(a.clauses, "material");
				if(!g || !mc)
				{
					record_error("actor @" + a.name + " is missing geometry or material; skipped");
					continue;
				}
				std::vector<double> local;
				geometry_tris(*g, local);
				std::vector<float> world;
				bake(a, local, world, true);
				add_triangles(world, material_of(mc->value), 0u);
			}
			else if(a.type == "model-light" || a.type == "rectangle-light" || a.type == "area-light")
			{
				std::vector<double> local;
				uint32_t mat;
				if(a.type == "model-light")
				{
					const Resource* g = ref(a, "geometry");
					if(!g)
					{
						throw std::runtime_error("model light @" + a.name + " has no geometry");
					}
					geometry_tris(*g, local);
					const SdlClause* mc = find(a.clauses, "material");
					mat = mc ? material_of(mc->value) : default_matte_index();
				}
				else
				{
					Resource rect;
					rect.type = "rectangle";
					rect.clauses = a.clauses;
					geometry_tris(rect, local);
					mat = absorber_index();
				}
				if(const SdlClause* bf = find(a.clauses, "back-face-emit"))
				{
					if(lower(bf->value) == "true")
					{
						throw std::runtime_error("back-face emission is not supported by the GPU renderer");
					}
				}
				for(const char* flag : {"directly-visible", "bsdf-sample", "direct-sample"})
				{
					if(const SdlClause* f = find(a.clauses, flag))
					{
						if(lower(f->value) == "false")
						{
							throw std::runtime_error(std::string(flag) + " = false is not supported by the GPU renderer");
						}
					}
				}
				std::vector<float> world;
				bake(a, local, world, true);
				EmitterRec e{};
				e.type = PG_EMITTER_TRIANGLES;
				desc.emitters.push_back(e);
				const uint32_t eid = static_cast<uint32_t>(desc.emitters.size());
				const double area = add_triangles(world, mat, eid);
				double rgb[3] = {1, 1, 1};
				if(a.type == "model-light")
				{
					if(const SdlClause* ee = find(a.clauses, "emitted-energy"))
					{
						image_rgb(*ee, rgb);
					}
					else
					{
						throw std::runtime_error("model light without emitted-energy (unit D65 default unsupported)");
					}
				}
				else
				{
					// radiance = putEnergy(color, watts) / (area * pi) (AAreaLight.cpp:57-58)
					double color[3] = {1, 1, 1};
					get_vec3(a.clauses, "color", color);
					const double watts = get_real(a.clauses, "watts", 100.0);
					const double energy = color_energy(color[0], color[1], color[2]);
					for(int k = 0; k < 3; ++k)
					{
						rgb[k] = energy > 0.0 ? color[k] / energy * watts / (area * kPiD) : 0.0;
					}
				}
				desc.emitters.back().r = static_cast<float>(rgb[0]);
				desc.emitters.back().g = static_cast<float>(rgb[1]);
				desc.emitters.back().b = static_cast<float>(rgb[2]);
			}
			else if(a.type == "image-dome")
			{
				const SdlClause* f = find(a.clauses, "image-file");
				if(!f)
				{
					throw std::runtime_error("image dome without image-file");
				}
				const std::string path = resolve_resource(f->value);
				HdrFrame img;
				if(!read_pfm(path, img))
				{
					throw std::runtime_error("cannot read dome image " + path + " (PFM only)");
				}
				if(img.width == 0 || img.height == 0 || img.rgb.size() != static_cast<std::size_t>(img.width) * img.height * 3)
				{
					throw std::runtime_error("dome image " + path + " is empty");
				}
				const double scale = get_real(a.clauses, "energy-scale", 1.0);
				desc.has_env = true;
				if(img.width == 1 && img.height == 1)
				{
					// constant environment
					for(int k = 0; k < 3; ++k) { desc.env_rgb[k] = static_cast<float>(img.rgb[k] * scale); }
				}
				else
				{
					// lat-long image, row 0 at the bottom (looking down), and the dome's rotation
					// (its scale has no effect, ADome.cpp:25-40)
					desc.env_width = img.width;
					desc.env_height = img.height;
					desc.env_image.resize(img.rgb.size());
					double mean[3] = {0, 0, 0};
					for(std::size_t k = 0; k < img.rgb.size(); ++k)
					{
						desc.env_image[k] = static_cast<float>(img.rgb[k] * scale);
						mean[k % 3] += desc.env_image[k];
					}
					for(int k = 0; k < 3; ++k) { desc.env_rgb[k] = static_cast<float>(mean[k] / (img.width * img.height)); }
					for(int c = 0; c < 3; ++c)
					{
						const double axis[3] = {c == 0 ? 1.0 : 0.0, c == 1 ? 1.0 : 0.0, c == 2 ? 1.0 : 0.0};
						double col[3];
						quat_rotate(a.rot, axis, col);
						for(int r = 0; r < 3; ++r) { desc.env_rot[3 * r + c] = static_cast<float>(col[r]); }
					}
				}
				for(int k = 0; k < 3; ++k) { dome_center[k] = a.pos[k]; }
				has_dome = true;
			}
			else
			{
				throw std::runtime_error("actor(" + a.type + ") is not supported by the GPU renderer");
			}
		}
		if(has_dome)
		{
			EmitterRec e{};
			e.type = PG_EMITTER_ENV;
			e.r = desc.env_rgb[0]; e.g = desc.env_rgb[1]; e.b = desc.env_rgb[2];
			desc.emitters.push_back(e);
			const float c[3] = {static_cast<float>(dome_center[0]), static_cast<float>(dome_center[1]), static_cast<float>(dome_center[2])};
			desc.env_area = dome_area(desc.tris, c);
			for(int k = 0; k < 3; ++k) { desc.env_center[k] = c[k]; }
		}
		if(desc.tris.empty())
		{
			throw std::runtime_error("the scene has no triangles");
		}
		const float p3[3] = {static_cast<float>(pos[0]), static_cast<float>(pos[1]), static_cast<float>(pos[2])};
		const float d3[3] = {static_cast<float>(dir[0]), static_cast<float>(dir[1]), static_cast<float>(dir[2])};
		const float u3[3] = {static_cast<float>(up[0]), static_cast<float>(up[1]), static_cast<float>(up[2])};
		desc.camera = make_camera(p3, d3, u3, static_cast<float>(fov), width, height, static_cast<float>(sensor_w));
		m_width = width;
		m_height = height;
	}
}

std::string Engine::resolve_resource(const std::string& identifier) const
{
	// SDL resource identifiers: ":rel/path" is relative to the scene's working directory,
	// "ext:/abs/path" is external (SdlResourceLocator.cpp:20-43, 190-210).
	if(identifier.rfind("ext:", 0) == 0) { return identifier.substr(4); }
	if(!identifier.empty() && identifier[0] == ':') { return m_working_dir + "/" + identifier.substr(1); }
	if(identifier.empty() || identifier[0] != '/') { return m_working_dir + "/" + identifier; }
	return identifier;
}

void Engine::set_dome_pdf(uint32_t mode)
{
	m_dome_pdf = mode;
	if(m_render)
	{
		m_render->scene->set_dome_exact(mode == 1u);
	}
}

void Engine::render()
{
	if(!m_render)
	{
		record_error("render: the scene was not updated successfully");
		return;
	}
	try
	{
		const auto t0 = std::chrono::steady_clock::now();
		const uint64_t wh = static_cast<uint64_t>(m_width) * m_height;
		// Progress is reported per chunk of samples; each chunk is at most 2^31 paths.
		uint32_t chunk = m_spp;
		const uint64_t max_chunk_spp = std::max<uint64_t>(1, (1ull << 31) / wh);
		if(chunk > max_chunk_spp) { chunk = static_cast<uint32_t>(max_chunk_spp); }
		m_work_total = m_spp;
		m_work_done = 0;
		{
			GuideParams g = m_render->scene->guiding();
			g.enabled = m_guiding;
			m_render->scene->set_guiding(g);
		}
		m_info = RenderInfo{0.0, 0, 0, 0, m_info.update_seconds, m_info.num_triangles};
		m_launches = 0;
		uint32_t done = 0;
		// progress points: a preview of the finished samples, an UPDATING region, the statistics
		begin_preview(*m_render);
		RenderProgress progress;
		progress.mutex = &m_render->frame_mutex;
		progress.preview_rgb = m_render->preview.get();
		progress.published = [&](unsigned long long finished, unsigned long long)
		{
			const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
			const double paths = static_cast<double>(wh) * done + static_cast<double>(finished);
			m_work_done = done + static_cast<uint64_t>(finished / wh);
			m_elapsed_ms = static_cast<uint64_t>(secs * 1000.0);
			m_samples_per_second = secs > 0.0 ? static_cast<float>(paths / secs) : 0.0f;
			push_region(false);
		};
		struct PreviewEnd
		{
			RenderObject& r;
			~PreviewEnd() { end_preview(r); }
		} preview_end{*m_render};
		while(done < m_spp)
		{
			const uint32_t n = std::min(chunk, m_spp - done);
			RenderParams p;
			p.width = m_width;
			p.height = m_height;
			p.spp = n;
			p.max_bounces = m_max_bounces;
			p.estimator = m_estimator;
			p.filter = m_render->filter;
			p.refine_mode = m_refine.refine_mode;
			p.refine_delta = m_refine.refine_delta;
			p.refine_iters = m_refine.refine_iters;
			p.seed = m_seed;
			p.first_sample = m_first_sample + m_render->samples;
			p.progress = &progress;
			const float ms = m_render->scene->render(p, m_render->film.get());
			m_render->samples += n;
			m_info.device_ms += ms;
			m_info.paths += wh * n;
			m_info.rays += m_render->scene->last_rays();
			m_info.shadow_rays += m_render->scene->last_shadow_rays();
			m_launches += m_render->scene->last_launches();
			done += n;
			m_work_done = done;
			const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
			m_elapsed_ms = static_cast<uint64_t>(secs * 1000.0);
			m_samples_per_second = secs > 0.0 ? static_cast<float>(static_cast<double>(wh) * done / secs) : 0.0f;
		}
	}
	catch(const std::exception& e)
	{
		record_error(std::string("render failed: ") + e.what());
	}
	push_region(true);
}

void Engine::push_region(bool finished)
{
	std::lock_guard<std::mutex> lock(m_region_mutex);
	if(!finished && m_regions.size() >= kMaxQueuedRegions)
	{
		return;
	}
	m_regions.push_back(RegionUpdate{0u, 0u, m_width, m_height, finished});
}

std::size_t Engine::poll_regions(RegionUpdate* out, std::size_t max)
{
	std::lock_guard<std::mutex> lock(m_region_mutex);
	std::size_t n = 0;
	while(n < max && !m_regions.empty())
	{
		out[n++] = m_regions.front();
		m_regions.pop_front();
	}
	return n;
}

std::size_t Engine::poll_merged_regions(RegionUpdate* out, std::size_t max)
{
	std::lock_guard<std::mutex> lock(m_region_mutex);
	if(max == 0 || m_regions.empty())
	{
		return 0;
	}
	out[0] = m_regions.back();
	m_regions.clear();
	return 1;
}

void Engine::profile(uint32_t mode, uint32_t spp, double out_stats[14])
{
	for(int k = 0; k < 14; ++k) { out_stats[k] = 0.0; }
	if(!m_render)
	{
		throw std::runtime_error("profile: the scene was not updated successfully");
	}
	DeviceBuffer<double> scratch(static_cast<std::size_t>(m_width) * m_height * kFilmChannels);
	PG_CUDA_CHECK(cudaMemsetAsync(scratch.get(), 0, scratch.bytes(), library_stream()));
	RenderParams p;
	p.width = m_width;
	p.height = m_height;
	p.spp = spp;
	p.max_bounces = m_max_bounces;
	p.estimator = m_estimator;
	p.filter = m_render->filter;
	p.refine_mode = m_refine.refine_mode;
	p.refine_delta = m_refine.refine_delta;
	p.refine_iters = m_refine.refine_iters;
	p.seed = m_seed + 0x9E3779B97F4A7C15ull;
	p.mode = mode;
	RenderScene& rs = *m_render->scene;
	const float ms = rs.render(p, scratch.get());
	for(int k = 0; k < 5; ++k) { out_stats[k] = rs.last_kernel_ms()[k]; }
	out_stats[5] = ms;
	out_stats[6] = static_cast<double>(m_width) * m_height * spp;
	out_stats[7] = static_cast<double>(rs.last_rays());
	out_stats[8] = static_cast<double>(rs.last_shadow_rays());
	out_stats[9] = static_cast<double>(rs.last_iterations());
	for(int k = 0; k < 4; ++k) { out_stats[10 + k] = static_cast<double>(rs.last_counts()[k]); }
}

AutotuneResult Engine::autotune(const char* cache_path, uint32_t flags)
{
	if(!m_render)
	{
		throw std::runtime_error("autotune: the scene was not updated successfully");
	}
	RenderParams p;
	p.width = m_width;
	p.height = m_height;
	p.spp = m_spp;
	p.max_bounces = m_max_bounces;
	p.estimator = m_estimator;
	p.filter = m_render->filter;
	p.refine_mode = m_refine.refine_mode;
	p.refine_delta = m_refine.refine_delta;
	p.refine_iters = m_refine.refine_iters;
	p.seed = m_seed + 0x632BE59BD9B4E019ull;
	return m_render->scene->autotune(p, (flags & 1u) != 0u, cache_path, (flags & 2u) != 0u);
}

void Engine::clear_film()
{
	if(m_render)
	{
		PG_CUDA_CHECK(cudaMemsetAsync(m_render->film.get(), 0, m_render->film.bytes(), library_stream()));
		PG_CUDA_CHECK(cudaStreamSynchronize(library_stream()));
		m_render->samples = 0;
	}
}

void Engine::get_render_dimension(uint32_t* w, uint32_t* h) const
{
	if(w) { *w = m_width; }
	if(h) { *h = m_height; }
}

void Engine::retrieve_frame(HdrFrame& frame) const
{
	peek_frame(0, 0, m_width, m_height, frame);
}

void Engine::peek_frame(uint32_t x, uint32_t y, uint32_t w, uint32_t h, HdrFrame& frame) const
{
	if(!m_render)
	{
		return;
	}
	const std::size_t pixels = static_cast<std::size_t>(m_width) * m_height;
	if(frame.width != m_width || frame.height != m_height || frame.rgb.size() != pixels * 3)
	{
		if(frame.width != 0 && (frame.width != m_width || frame.height != m_height))
		{
			// the reference warns and leaves the frame untouched (HdrRgbFilm.cpp:167-178)
			return;
		}
		frame.width = m_width;
		frame.height = m_height;
		frame.rgb.assign(pixels * 3, 0.0f);
	}
	develop_frame(*m_render, frame.rgb.data(), x, y, w, h);
}

void Engine::get_progress(uint64_t* total, uint64_t* done, uint64_t* elapsed_ms) const
{
	if(total) { *total = m_work_total.load(); }
	if(done) { *done = m_work_done.load(); }
	if(elapsed_ms) { *elapsed_ms = m_elapsed_ms.load(); }
}

void Engine::get_statistics(float* percentage, float* samples_per_second) const
{
	const uint64_t total = m_work_total.load();
	if(percentage) { *percentage = total ? 100.0f * static_cast<float>(m_work_done.load()) / static_cast<float>(total) : 0.0f; }
	if(samples_per_second) { *samples_per_second = m_samples_per_second.load(); }
}

bool write_pfm(const std::string& path, const HdrFrame& frame)
{
	FILE* f = std::fopen(path.c_str(), "wb");
	if(!f)
	{
		return false;
	}
	std::fprintf(f, "PF\n%u %u\n-1.0\n", frame.width, frame.height);
	// PFM scanlines run bottom to top, which is the frame's own row order.
	const bool ok = std::fwrite(frame.rgb.data(), sizeof(float), frame.rgb.size(), f) == frame.rgb.size();
	std::fclose(f);
	return ok;
}

bool read_pfm(const std::string& path, HdrFrame& frame)
{
	std::ifstream in(path, std::ios::binary);
	if(!in)
	{
		return false;
	}
	std::string magic;
	in >> magic;
	if(magic != "PF" && magic != "Pf")
	{
		return false;
	}
	long long w = 0, h = 0;
	double scale = 0.0;
	in >> w >> h >> scale;
	in.get();
	if(!in || w < 0 || h < 0 || w > 0x7FFFFFFFll || h > 0x7FFFFFFFll || !std::isfinite(scale) || scale == 0.0)
	{
		return false;
	}
	const int channels = magic == "PF" ? 3 : 1;
	// the header's size must be backed by the bytes that follow it (checked before allocating)
	const std::streamoff body_begin = in.tellg();
	in.seekg(0, std::ios::end);
	const std::streamoff body_bytes = in.tellg() - body_begin;
	in.seekg(body_begin);
	const unsigned long long needed = static_cast<unsigned long long>(w) * static_cast<unsigned long long>(h) * channels * 4ull;
	if(body_begin < 0 || body_bytes < 0 || static_cast<unsigned long long>(body_bytes) < needed)
	{
		return false;
	}
	std::vector<float> data(static_cast<std::size_t>(w) * static_cast<std::size_t>(h) * channels);
	in.read(reinterpret_cast<char*>(data.data()), static_cast<std::streamsize>(data.size() * sizeof(float)));
	if(!in)
	{
		return false;
	}
	if(scale > 0.0)
	{
		for(float& v : data)
		{
			uint32_t u;
			std::memcpy(&u, &v, 4);
			u = __builtin_bswap32(u);
			std::memcpy(&v, &u, 4);
		}
	}
	frame.width = static_cast<uint32_t>(w);
	frame.height = static_cast<uint32_t>(h);
	frame.rgb.resize(static_cast<std::size_t>(w) * static_cast<std::size_t>(h) * 3);
	for(std::size_t i = 0; i < static_cast<std::size_t>(w) * static_cast<std::size_t>(h); ++i)
	{
		for(int c = 0; c < 3; ++c)
		{
			frame.rgb[3 * i + c] = data[i * channels + (channels == 3 ? c : 0)];
		}
	}
	return true;
}

EngineSettings& engine_settings()
{
	static EngineSettings settings;
	return settings;
}

bool load_engine_settings(const std::string& path, EngineSettings& out)
{
	std::ifstream in(path);
	if(!in)
	{
		return false;
	}
	auto trim = [](const std::string& x)
	{
		const auto b = x.find_first_not_of(" \t\r");
		const auto e = x.find_last_not_of(" \t\r");
		return b == std::string::npos ? std::string() : x.substr(b, e - b + 1);
	};
	std::string line;
	while(std::getline(in, line))
	{
		const auto eq = line.find('=');
		if(eq == std::string::npos)
		{
			continue;
		}
		const std::string key = trim(line.substr(0, eq)), value = trim(line.substr(eq + 1));
		try
		{
			if(key == "RefineMode")
			{
				if(value == "manual") { out.refine_mode = 0; }
				else if(value == "empirical") { out.refine_mode = 1; }
				else if(value == "iterative") { out.refine_mode = 2; }
			}
			else if(key == "SelfIntersectDelta")
			{
				out.refine_delta = std::stof(value);
			}
			else if(key == "NumIterativeSurfaceRefinements")
			{
				out.refine_iters = std::max<uint32_t>(1u, static_cast<uint32_t>(std::stoul(value)));
			}
		}
		catch(const std::exception&)
		{
			// a malformed number keeps the previous value, as an absent key would
		}
	}
	return true;
}

}// end namespace pg
