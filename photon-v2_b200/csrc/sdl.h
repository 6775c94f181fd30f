// Parser for Photon's scene description language (SDL 1.1 command syntax).
//
// Grammar handled (the reference's SdlCommandParser, Engine/Source/SDL/SdlCommandParser.cpp:84-560,
// and SdlInlinePacketInterface, Engine/Source/SDL/SdlInlinePacketInterface.cpp:48-245):
//   text      := commands separated by ';', '//' starts a comment that runs to the end of line
//   directive := '#' ...                                   (e.g. `#version 1.1.0`)
//   load      := category '(' type ')' '@' name '=' clause*
//   execution := [category '(' type ')' '.'] func '(' '@' target ')' '=' clause*
//   clause    := '[' type name[':' tag] value ']'
//   value     := token | "quoted text" | '{' array '}' | '@' reference
// Commands may arrive split across any number of fragments (phEnterCommand streams them).
#pragma once

#include <functional>
#include <string>
#include <string_view>
#include <vector>

namespace pg
{

struct SdlClause
{
	std::string type;
	std::string name;
	std::string value;
	bool        is_reference = false;
};

struct SdlCommand
{
	enum class Kind { Load, Execution, Directive };

	Kind        kind = Kind::Load;
	std::string category;   // e.g. "geometry" (may be empty for an execution)
	std::string type;       // e.g. "triangle-mesh"
	std::string name;       // resource name of a load, target name of an execution
	std::string function;   // execution function name, e.g. "translate"
	std::string directive;  // directive text without '#'
	std::vector<SdlClause> clauses;

	const SdlClause* find(std::string_view clause_name) const;
};

class SdlParser
{
public:
	using Sink = std::function<void(SdlCommand&&)>;

	// Feeds a fragment; every command completed by it is parsed and passed to `sink`.
	// Malformed commands throw std::runtime_error after the rest of the fragment is buffered.
	void feed(std::string_view fragment, const Sink& sink);

	// Parses one complete command (no trailing ';').
	static SdlCommand parse_command(std::string_view command);

	std::size_t num_errors() const { return m_num_errors; }
	const std::vector<std::string>& errors() const { return m_errors; }

private:
	std::string m_pending;
	bool        m_in_comment = false;
	std::size_t m_num_errors = 0;
	std::vector<std::string> m_errors;
};

// Value helpers.
std::vector<double> sdl_numbers(std::string_view value);
// Vector3 array of the form `"x y z" "x y z" ...` (content of the braces).
std::vector<float> sdl_vector3_array(std::string_view value);

}// end namespace pg
