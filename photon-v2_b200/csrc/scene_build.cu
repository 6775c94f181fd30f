#include "scene_build.h"

#include <algorithm>
#include <cmath>
#include <string>

namespace pg
{

void checked_resolution(double width, double height, const char* who, uint32_t* out_width, uint32_t* out_height)
{
	auto whole = [](double v) { return std::isfinite(v) && v >= 1.0 && v <= 2147483648.0 && v == std::floor(v); };
	if(!whole(width) || !whole(height) || width * height > 2147483648.0)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, std::string(who) + ": the resolution must be two whole numbers of at least 1 "
		                                     "with at most 2^31 pixels in all");
	}
	*out_width = static_cast<uint32_t>(width);
	*out_height = static_cast<uint32_t>(height);
}

Camera make_camera(const float pos[3], const float dir[3], const float up[3], float fov_degrees,
                   uint32_t width, uint32_t height, float sensor_width_mm)
{
	// Basis in double as the reference computes it (Vector3D), then stored as float.
	double z[3] = {-dir[0], -dir[1], -dir[2]};
	const double zl = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
	if(zl > 0.001)
	{
		for(double& c : z) { c /= zl; }
	}
	else
	{
		z[0] = 0.0; z[1] = 0.0; z[2] = 1.0;
	}
	auto cross = [](const double a[3], const double b[3], double out[3])
	{
		out[0] = a[1] * b[2] - a[2] * b[1];
		out[1] = a[2] * b[0] - a[0] * b[2];
		out[2] = a[0] * b[1] - a[1] * b[0];
	};
	const double u[3] = {up[0], up[1], up[2]};
	double x[3], y[3];
	cross(u, z, x);
	cross(z, x, y);
	const double xl = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
	if(xl > 0.001)
	{
		const double yl = std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
		for(int i = 0; i < 3; ++i) { x[i] /= xl; y[i] /= yl; }
	}
	else
	{
		// Recover with +x as right or +y as up (OrientedRasterObserver.cpp:79-96).
		const double ex[3] = {1, 0, 0}, ey[3] = {0, 1, 0};
		if(std::fabs(z[0]) < std::fabs(z[1]))
		{
			cross(z, ex, y);
			const double yl = std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
			for(double& c : y) { c /= yl; }
			cross(y, z, x);
			const double xl2 = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
			for(double& c : x) { c /= xl2; }
		}
		else
		{
			cross(ey, z, x);
			const double xl2 = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
			for(double& c : x) { c /= xl2; }
			cross(z, x, y);
			const double yl = std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
			for(double& c : y) { c /= yl; }
		}
	}

	Camera c{};
	for(int i = 0; i < 3; ++i)
	{
		c.pos[i] = pos[i];
		c.axis_x[i] = static_cast<float>(x[i]);
		c.axis_y[i] = static_cast<float>(y[i]);
		c.axis_z[i] = static_cast<float>(z[i]);
	}
	const double aspect = static_cast<double>(width) / static_cast<double>(height);
	const double sensor_w = sensor_width_mm / 1000.0;
	const double sensor_h = (sensor_width_mm / aspect) / 1000.0;
	const double half_fov = fov_degrees * 3.14159265358979323846 / 180.0 * 0.5;
	c.sensor_w = static_cast<float>(sensor_w);
	c.sensor_h = static_cast<float>(sensor_h);
	c.sensor_offset = static_cast<float>((sensor_w * 0.5) / std::tan(half_fov));
	c.width = width;
	c.height = height;
	return c;
}

Material make_matte(float r, float g, float b)
{
	Material m{};
	m.type = PG_MAT_MATTE;
	m.cr = r; m.cg = g; m.cb = b;
	return m;
}

Material make_conductor(float roughness, float f0r, float f0g, float f0b)
{
	Material m{};
	m.type = PG_MAT_CONDUCTOR;
	m.cr = f0r; m.cg = f0g; m.cb = f0b;
	const float alpha = roughness * roughness;
	m.alpha = alpha > 0.001f ? alpha : 0.001f;
	return m;
}

Material make_dielectric(float roughness, float ior_outer, float ior_inner)
{
	Material m{};
	m.type = PG_MAT_DIELECTRIC;
	const float alpha = roughness * roughness;
	m.alpha = alpha > 0.001f ? alpha : 0.001f;
	m.ior_outer = ior_outer;
	m.ior_inner = ior_inner;
	return m;
}

namespace
{
// Energy of the seven Smits basis spectra (white, cyan, magenta, yellow, red, green, blue) as the
// reference's upsampling sums them, obtained by running its estimate_color_energy on the seven
// basis colours. With Smits' decomposition (min * white + (mid - min) * secondary +
// (max - mid) * primary) they give the energy of any colour.
constexpr double kSmitsEnergy[7] = {
	0.999678004, 0.539849638, 0.734938899, 0.704456255, 0.454419964, 0.258257833, 0.302870461};
}

double color_energy(double r, double g, double b)
{
	const double W = kSmitsEnergy[0], C = kSmitsEnergy[1], M = kSmitsEnergy[2], Y = kSmitsEnergy[3];
	const double R = kSmitsEnergy[4], G = kSmitsEnergy[5], B = kSmitsEnergy[6];
	double e;
	if(r <= g && r <= b)
	{
		e = r * W + (g <= b ? (g - r) * C + (b - g) * B : (b - r) * C + (g - b) * G);
	}
	else if(g <= r && g <= b)
	{
		e = g * W + (r <= b ? (r - g) * M + (b - r) * B : (b - g) * M + (r - b) * R);
	}
	else
	{
		e = b * W + (r <= g ? (r - b) * Y + (g - r) * G : (g - b) * Y + (r - g) * R);
	}
	return e > 0.0 ? e : 0.0;
}

double dome_area(const std::vector<float>& tris, const float center[3])
{
	double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
	for(std::size_t i = 0; i + 2 < tris.size(); i += 3)
	{
		for(int a = 0; a < 3; ++a)
		{
			lo[a] = std::min(lo[a], static_cast<double>(tris[i + a]));
			hi[a] = std::max(hi[a], static_cast<double>(tris[i + a]));
		}
	}
	double radius = 1.0;
	for(int k = 0; k < 8; ++k)
	{
		const double v[3] = {(k & 1) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1], (k & 4) ? hi[2] : lo[2]};
		const double dx = v[0] - center[0], dy = v[1] - center[1], dz = v[2] - center[2];
		radius = std::max(radius, std::sqrt(dx * dx + dy * dy + dz * dz) * 1.01);
	}
	return 4.0 * 3.14159265358979323846 * radius * radius;
}

}// end namespace pg
