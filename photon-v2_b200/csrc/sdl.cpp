#include "sdl.h"

#include <cctype>
#include <charconv>
#include <cstdlib>
#include <stdexcept>

namespace pg
{
namespace
{

std::string_view trim(std::string_view s)
{
	std::size_t b = 0, e = s.size();
	while(b < e && std::isspace(static_cast<unsigned char>(s[b]))) { ++b; }
	while(e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) { --e; }
	return s.substr(b, e - b);
}

// Splits on whitespace; text inside an enclosure pair is one token with the enclosure removed.
std::vector<std::string> tokenize(std::string_view s, const char* openers, const char* closers)
{
	std::vector<std::string> out;
	std::size_t i = 0;
	const std::string_view open(openers), close(closers);
	while(i < s.size())
	{
		while(i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) { ++i; }
		if(i >= s.size())
		{
			break;
		}
		const std::size_t k = open.find(s[i]);
		if(k != std::string_view::npos)
		{
			const char closer = close[k];
			const std::size_t end = s.find(closer, i + 1);
			if(end == std::string_view::npos)
			{
				throw std::runtime_error("unterminated enclosure in: " + std::string(s.substr(i, 40)));
			}
			out.emplace_back(s.substr(i + 1, end - i - 1));
			i = end + 1;
		}
		else
		{
			std::size_t j = i;
			while(j < s.size() && !std::isspace(static_cast<unsigned char>(s[j])) && open.find(s[j]) == std::string_view::npos)
			{
				++j;
			}
			out.emplace_back(s.substr(i, j - i));
			i = j;
		}
	}
	return out;
}

// Clause strings: the contents of every [...] group.
std::vector<std::string_view> clause_strings(std::string_view data)
{
	std::vector<std::string_view> out;
	std::size_t i = 0;
	while(i < data.size())
	{
		const std::size_t b = data.find('[', i);
		if(b == std::string_view::npos)
		{
			if(!trim(data.substr(i)).empty())
			{
				throw std::runtime_error("syntax error: text outside of clauses");
			}
			break;
		}
		if(!trim(data.substr(i, b - i)).empty())
		{
			throw std::runtime_error("syntax error: text outside of clauses");
		}
		// a ']' inside quotes or braces does not close the clause
		std::size_t j = b + 1;
		char enclosure = 0;
		for(; j < data.size(); ++j)
		{
			const char c = data[j];
			if(enclosure)
			{
				if((enclosure == '"' && c == '"') || (enclosure == '{' && c == '}'))
				{
					enclosure = 0;
				}
			}
			else if(c == '"' || c == '{')
			{
				enclosure = c;
			}
			else if(c == ']')
			{
				break;
			}
		}
		if(j >= data.size())
		{
			throw std::runtime_error("syntax error: unterminated clause");
		}
		out.push_back(data.substr(b + 1, j - b - 1));
		i = j + 1;
	}
	return out;
}

SdlClause parse_clause(std::string_view s)
{
	const auto tokens = tokenize(s, "\"{", "\"}");
	if(tokens.size() < 2)
	{
		throw std::runtime_error("syntax error: incomplete clause [" + std::string(s) + "]");
	}
	SdlClause c;
	c.type = tokens[0];
	const auto colon = tokens[1].find(':');
	c.name = colon == std::string::npos ? tokens[1] : tokens[1].substr(0, colon);
	if(tokens.size() == 2)
	{
		return c;
	}
	if(tokens.size() == 3)
	{
		if(!tokens[2].empty() && tokens[2].front() == '@' && s.find("\"@") == std::string_view::npos)
		{
			c.is_reference = true;
			c.value = tokens[2].substr(1);
		}
		else
		{
			c.value = tokens[2];
		}
		return c;
	}
	if(tokens.size() == 4 && tokens[2] == "@")
	{
		c.is_reference = true;
		c.value = tokens[3];
		return c;
	}
	throw std::runtime_error("syntax error: too many tokens in clause [" + std::string(s) + "]");
}

// "name(arg)" -> (name, arg)
bool split_call(std::string_view s, std::string& name, std::string& arg)
{
	const auto lp = s.find('(');
	const auto rp = s.rfind(')');
	if(lp == std::string_view::npos || rp == std::string_view::npos || rp < lp)
	{
		return false;
	}
	name = std::string(trim(s.substr(0, lp)));
	arg = std::string(trim(s.substr(lp + 1, rp - lp - 1)));
	return true;
}

std::string strip_reference(std::string s)
{
	s = std::string(trim(s));
	if(!s.empty() && s.front() == '@')
	{
		s = s.substr(1);
	}
	if(s.size() >= 2 && s.front() == '"' && s.back() == '"')
	{
		s = s.substr(1, s.size() - 2);
	}
	return s;
}

}// end anonymous namespace

const SdlClause* SdlCommand::find(std::string_view clause_name) const
{
	for(const auto& c : clauses)
	{
		if(c.name == clause_name)
		{
			return &c;
		}
	}
	return nullptr;
}

SdlCommand SdlParser::parse_command(std::string_view command)
{
	SdlCommand cmd;
	const std::string_view text = trim(command);
	if(!text.empty() && text.front() == '#')
	{
		cmd.kind = SdlCommand::Kind::Directive;
		cmd.directive = std::string(trim(text.substr(1)));
		return cmd;
	}
	const auto eq = text.find('=');
	if(eq == std::string_view::npos)
	{
		throw std::runtime_error("syntax error: data command requires an assignment operator");
	}
	const std::string_view header = trim(text.substr(0, eq));
	const std::string_view data = text.substr(eq + 1);

	const auto at = header.find('@');
	const auto dot = header.substr(0, at).find(").");
	std::string first, first_arg;
	if(dot != std::string_view::npos)
	{
		// category(type).func(@target)
		if(!split_call(header.substr(0, dot + 1), cmd.category, cmd.type))
		{
			throw std::runtime_error("syntax error: bad command header");
		}
		std::string arg;
		if(!split_call(header.substr(dot + 2), cmd.function, arg))
		{
			throw std::runtime_error("syntax error: bad execution header");
		}
		cmd.kind = SdlCommand::Kind::Execution;
		cmd.name = strip_reference(arg);
	}
	else if(at != std::string_view::npos && header.find(')') < at)
	{
		const std::string_view call = trim(header.substr(0, at));
		const std::string_view after_at = trim(header.substr(at));
		if(call.back() == ')' && after_at.find(')') == std::string_view::npos)
		{
			// category(type) @name
			if(!split_call(call, cmd.category, cmd.type))
			{
				throw std::runtime_error("syntax error: bad command header");
			}
			cmd.kind = SdlCommand::Kind::Load;
			cmd.name = strip_reference(std::string(after_at));
		}
		else
		{
			std::string arg;
			if(!split_call(header, cmd.function, arg))
			{
				throw std::runtime_error("syntax error: bad execution header");
			}
			cmd.kind = SdlCommand::Kind::Execution;
			cmd.name = strip_reference(arg);
		}
	}
	else
	{
		// func(@target)
		std::string arg;
		if(!split_call(header, cmd.function, arg))
		{
			throw std::runtime_error("syntax error: unrecognised command header");
		}
		cmd.kind = SdlCommand::Kind::Execution;
		cmd.name = strip_reference(arg);
	}
	for(const auto cs : clause_strings(data))
	{
		cmd.clauses.push_back(parse_clause(cs));
	}
	return cmd;
}

void SdlParser::feed(std::string_view fragment, const Sink& sink)
{
	std::string error;
	std::size_t i = 0;
	while(i < fragment.size())
	{
		if(m_in_comment)
		{
			const auto nl = fragment.find('\n', i);
			if(nl == std::string_view::npos)
			{
				return;
			}
			m_in_comment = false;
			i = nl + 1;
			continue;
		}
		const auto k = fragment.find_first_of("/;", i);
		if(k == std::string_view::npos)
		{
			m_pending.append(fragment.substr(i));
			break;
		}
		if(fragment[k] == '/')
		{
			if(k + 1 < fragment.size() && fragment[k + 1] == '/')
			{
				m_pending.append(fragment.substr(i, k - i));
				m_in_comment = true;
				i = k + 2;
			}
			else
			{
				m_pending.append(fragment.substr(i, k - i + 1));
				i = k + 1;
			}
			continue;
		}
		// ';' completes a command
		m_pending.append(fragment.substr(i, k - i));
		i = k + 1;
		const std::string command = std::move(m_pending);
		m_pending.clear();
		if(trim(command).empty())
		{
			continue;
		}
		try
		{
			sink(parse_command(command));
		}
		catch(const std::exception& e)
		{
			++m_num_errors;
			const std::string shortened = std::string(trim(command).substr(0, 64));
			m_errors.push_back(std::string(e.what()) + " (parsing <" + shortened + ">)");
			if(error.empty())
			{
				error = m_errors.back();
			}
		}
	}
	if(!error.empty())
	{
		throw std::runtime_error(error);
	}
}

std::vector<double> sdl_numbers(std::string_view value)
{
	std::vector<double> out;
	for(const auto& tok : tokenize(value, "\"", "\""))
	{
		for(const auto& t : tokenize(tok, "", ""))
		{
			char* end = nullptr;
			const double v = std::strtod(t.c_str(), &end);
			if(end == t.c_str())
			{
				throw std::runtime_error("not a number: " + t);
			}
			out.push_back(v);
		}
	}
	return out;
}

std::vector<float> sdl_vector3_array(std::string_view value)
{
	std::vector<float> out;
	const char* p = value.data();
	const char* const end = value.data() + value.size();
	// Each element is a quoted "x y z" triple; parse numbers straight from the text (the arrays
	// of large meshes run to hundreds of megabytes).
	while(p < end)
	{
		while(p < end && *p != '"') { ++p; }
		if(p >= end)
		{
			break;
		}
		++p;
		const char* q = p;
		while(q < end && *q != '"') { ++q; }
		if(q >= end)
		{
			throw std::runtime_error("unterminated vector3 in array");
		}
		float xyz[3];
		int n = 0;
		const char* s = p;
		while(s < q && n < 3)
		{
			while(s < q && std::isspace(static_cast<unsigned char>(*s))) { ++s; }
			if(s >= q)
			{
				break;
			}
			auto [ptr, ec] = std::from_chars(s, q, xyz[n]);
			if(ec != std::errc())
			{
				throw std::runtime_error("bad number in vector3 array");
			}
			s = ptr;
			++n;
		}
		if(n == 1)
		{
			xyz[1] = xyz[2] = xyz[0];
		}
		else if(n != 3)
		{
			throw std::runtime_error("vector3 needs 1 or 3 numbers");
		}
		out.insert(out.end(), xyz, xyz + 3);
		p = q + 1;
	}
	return out;
}

}// end namespace pg
