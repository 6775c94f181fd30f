// PLY reader for triangle meshes (see ply.h).
#include "ply.h"

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <sstream>
#include <stdexcept>

namespace pg
{
namespace
{

enum class PlyType { I8, U8, I16, U16, I32, U32, F32, F64 };

PlyType parse_type(const std::string& t)
{
	if(t == "char" || t == "int8") { return PlyType::I8; }
	if(t == "uchar" || t == "uint8") { return PlyType::U8; }
	if(t == "short" || t == "int16") { return PlyType::I16; }
	if(t == "ushort" || t == "uint16") { return PlyType::U16; }
	if(t == "int" || t == "int32") { return PlyType::I32; }
	if(t == "uint" || t == "uint32") { return PlyType::U32; }
	if(t == "float" || t == "float32") { return PlyType::F32; }
	if(t == "double" || t == "float64") { return PlyType::F64; }
	throw std::runtime_error("PLY: unknown property type " + t);
}

std::size_t type_size(PlyType t)
{
	switch(t)
	{
	case PlyType::I8: case PlyType::U8: return 1;
	case PlyType::I16: case PlyType::U16: return 2;
	case PlyType::I32: case PlyType::U32: case PlyType::F32: return 4;
	case PlyType::F64: return 8;
	}
	return 0;
}

struct Property
{
	std::string name;
	bool is_list = false;
	PlyType count_type = PlyType::U8;
	PlyType type = PlyType::F32;
};

struct Element
{
	std::string name;
	uint64_t count = 0;
	std::vector<Property> props;
};

// One binary value, byte-swapped for big-endian files.
double read_value(const unsigned char* p, PlyType t, bool swap)
{
	unsigned char b[8];
	const std::size_t n = type_size(t);
	std::memcpy(b, p, n);
	if(swap)
	{
		std::reverse(b, b + n);
	}
	switch(t)
	{
	case PlyType::I8: { int8_t v; std::memcpy(&v, b, 1); return v; }
	case PlyType::U8: { uint8_t v; std::memcpy(&v, b, 1); return v; }
	case PlyType::I16: { int16_t v; std::memcpy(&v, b, 2); return v; }
	case PlyType::U16: { uint16_t v; std::memcpy(&v, b, 2); return v; }
	case PlyType::I32: { int32_t v; std::memcpy(&v, b, 4); return v; }
	case PlyType::U32: { uint32_t v; std::memcpy(&v, b, 4); return v; }
	case PlyType::F32: { float v; std::memcpy(&v, b, 4); return v; }
	case PlyType::F64: { double v; std::memcpy(&v, b, 8); return v; }
	}
	return 0.0;
}

// Sequential reader over the body: binary (with byte order) or whitespace-separated ASCII.
class BodyReader
{
public:
	BodyReader(std::vector<char> data, bool ascii, bool swap) : m_data(std::move(data)), m_ascii(ascii), m_swap(swap)
	{
		m_data.push_back('\0');   // strtod / strtoll stop at the terminator
	}

	double next(PlyType t)
	{
		if(m_ascii)
		{
			const char* begin = m_data.data() + m_pos;
			char* end = nullptr;
			const double v = (t == PlyType::F32 || t == PlyType::F64) ? std::strtod(begin, &end)
			                                                         : static_cast<double>(std::strtoll(begin, &end, 10));
			if(end == begin)
			{
				throw std::runtime_error("PLY: truncated or malformed ASCII body");
			}
			m_pos = static_cast<std::size_t>(end - m_data.data());
			return v;
		}
		const std::size_t n = type_size(t);
		if(m_pos + n > m_data.size() - 1)
		{
			throw std::runtime_error("PLY: truncated binary body");
		}
		const double v = read_value(reinterpret_cast<const unsigned char*>(m_data.data() + m_pos), t, m_swap);
		m_pos += n;
		return v;
	}

private:
	std::vector<char> m_data;
	std::size_t m_pos = 0;
	bool m_ascii;
	bool m_swap;
};

}// end anonymous namespace

PlyMesh read_ply(const std::string& path)
{
	std::ifstream in(path, std::ios::binary);
	if(!in)
	{
		throw std::runtime_error("cannot open PLY file " + path);
	}
	auto next_line = [&](std::string& line) -> bool
	{
		if(!std::getline(in, line))
		{
			return false;
		}
		if(!line.empty() && line.back() == '\r')
		{
			line.pop_back();
		}
		return true;
	};

	std::string line;
	if(!next_line(line) || line != "ply")
	{
		throw std::runtime_error("not a PLY file: " + path);
	}
	std::string format;
	std::vector<Element> elements;
	bool header_done = false;
	while(next_line(line))
	{
		std::istringstream ls(line);
		std::string word;
		ls >> word;
		if(word == "format")
		{
			std::string version;
			ls >> format >> version;
		}
		else if(word == "element")
		{
			Element e;
			ls >> e.name >> e.count;
			elements.push_back(e);
		}
		else if(word == "property")
		{
			if(elements.empty())
			{
				throw std::runtime_error("PLY: property before any element");
			}
			Property p;
			std::string t;
			ls >> t;
			if(t == "list")
			{
				std::string ct, vt;
				ls >> ct >> vt >> p.name;
				p.is_list = true;
				p.count_type = parse_type(ct);
				p.type = parse_type(vt);
			}
			else
			{
				p.type = parse_type(t);
				ls >> p.name;
			}
			elements.back().props.push_back(p);
		}
		else if(word == "end_header")
		{
			header_done = true;
			break;
		}
		// comment, obj_info and blank lines carry nothing needed here
	}
	if(!header_done)
	{
		throw std::runtime_error("PLY: no end_header");
	}
	const bool ascii = format == "ascii";
	const bool big = format == "binary_big_endian";
	if(!ascii && !big && format != "binary_little_endian")
	{
		throw std::runtime_error("PLY: unknown format " + format);
	}

	const Element* vertex = nullptr;
	const Element* face = nullptr;
	for(const Element& e : elements)
	{
		if(e.name == "vertex") { vertex = &e; }
		if(e.name == "face") { face = &e; }
	}
	if(!vertex || !face)
	{
		throw std::runtime_error("PLY: needs a vertex and a face element");
	}
	int ix = -1, iy = -1, iz = -1, inx = -1, iny = -1, inz = -1, iidx = -1;
	for(std::size_t k = 0; k < vertex->props.size(); ++k)
	{
		const std::string& n = vertex->props[k].name;
		if(n == "x") { ix = static_cast<int>(k); }
		if(n == "y") { iy = static_cast<int>(k); }
		if(n == "z") { iz = static_cast<int>(k); }
		if(n == "nx") { inx = static_cast<int>(k); }
		if(n == "ny") { iny = static_cast<int>(k); }
		if(n == "nz") { inz = static_cast<int>(k); }
	}
	for(std::size_t k = 0; k < face->props.size(); ++k)
	{
		const Property& p = face->props[k];
		if(p.is_list && (p.name == "vertex_indices" || p.name == "vertex_index"))
		{
			iidx = static_cast<int>(k);
		}
	}
	if(face < vertex)
	{
		// faces are resolved to positions while they are read
		throw std::runtime_error("PLY: the face element must follow the vertex element");
	}
	if(ix < 0 || iy < 0 || iz < 0)
	{
		throw std::runtime_error("PLY: the vertex element needs x, y and z");
	}
	if(iidx < 0)
	{
		throw std::runtime_error("PLY: the face element needs a vertex_indices list");
	}
	if(face->props[iidx].type == PlyType::F32 || face->props[iidx].type == PlyType::F64)
	{
		throw std::runtime_error("PLY: vertex indices must be integers");
	}

	std::vector<char> body((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
	// Every row takes at least a known number of bytes (binary: its scalars and list counts; ASCII:
	// one character and a separator per value), so element counts the body cannot hold are
	// rejected before anything is sized by them.
	long double min_bytes = 0.0L;
	for(const Element& e : elements)
	{
		if(e.props.empty() && e.count > 0)
		{
			// rows of no bytes: the count would drive a loop that reads nothing
			throw std::runtime_error("PLY: element '" + e.name + "' has rows but no properties");
		}
		uint64_t row = 0;
		for(const Property& p : e.props)
		{
			row += ascii ? 2u : type_size(p.is_list ? p.count_type : p.type);
		}
		min_bytes += static_cast<long double>(e.count) * static_cast<long double>(row);
	}
	if(min_bytes > static_cast<long double>(body.size()) + 1.0L)
	{
		throw std::runtime_error("PLY: truncated body (the header's element counts need more bytes than the file holds)");
	}
	BodyReader reader(std::move(body), ascii, big);

	PlyMesh mesh;
	mesh.has_normals = inx >= 0 && iny >= 0 && inz >= 0;
	std::vector<double> positions;
	for(const Element& e : elements)
	{
		const bool is_vertex = &e == vertex, is_face = &e == face;
		if(is_vertex)
		{
			positions.resize(3 * e.count);
		}
		if(is_face)
		{
			mesh.tris.reserve(9 * e.count);
		}
		for(uint64_t row = 0; row < e.count; ++row)
		{
			for(std::size_t k = 0; k < e.props.size(); ++k)
			{
				const Property& p = e.props[k];
				if(!p.is_list)
				{
					const double v = reader.next(p.type);
					if(is_vertex)
					{
						if(static_cast<int>(k) == ix) { positions[3 * row + 0] = v; }
						if(static_cast<int>(k) == iy) { positions[3 * row + 1] = v; }
						if(static_cast<int>(k) == iz) { positions[3 * row + 2] = v; }
					}
					continue;
				}
				const double count = reader.next(p.count_type);
				if(is_face && static_cast<int>(k) == iidx)
				{
					if(count != 3.0)
					{
						throw std::runtime_error("PLY: every face must have exactly 3 vertex indices "
						                         "(polygons of other sizes are not supported, as in the reference)");
					}
					for(int c = 0; c < 3; ++c)
					{
						const double idx = reader.next(p.type);
						if(idx < 0.0 || idx >= static_cast<double>(vertex->count))
						{
							throw std::runtime_error("PLY: vertex index out of range");
						}
						const std::size_t vi = static_cast<std::size_t>(idx);
						mesh.tris.insert(mesh.tris.end(), positions.begin() + 3 * vi, positions.begin() + 3 * vi + 3);
					}
				}
				else
				{
					for(uint64_t c = 0; c < static_cast<uint64_t>(count); ++c)
					{
						reader.next(p.type);
					}
				}
			}
		}
	}
	return mesh;
}

}// end namespace pg
