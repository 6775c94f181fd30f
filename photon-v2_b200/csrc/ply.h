// Triangle meshes from .ply files, for SDL's geometry(ply) [PRI ply-file ...] (the reference's
// GPlyPolygonMesh, Engine/Source/Actor/Geometry/GPlyPolygonMesh.cpp:68-200 over DataIO/PlyFile).
#pragma once

#include <string>
#include <vector>

namespace pg
{

struct PlyMesh
{
	std::vector<double> tris;    // [n][3][3] vertex positions of every face, in face order
	bool has_normals = false;    // the vertex element carries nx, ny, nz
};

// Reads format ascii / binary_little_endian / binary_big_endian 1.0: the vertex element's x, y, z
// (any scalar type) and the face element's vertex_indices (or vertex_index) lists, which must all
// have 3 entries, as the reference requires. Other elements and properties are skipped. Throws
// std::runtime_error with the reason on malformed input.
PlyMesh read_ply(const std::string& path);

}// end namespace pg
