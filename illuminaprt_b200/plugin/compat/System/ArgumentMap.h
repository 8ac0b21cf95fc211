// Replacement for the reference's System/ArgumentMap.h, found first on the
// include path when the engine headers are compiled here (the GPU space plug-in
// and the CPU checker built from the reference sources).
//
// Why: the reference's ArgumentMap (Core/System/ArgumentMap.h:243-258)
// returns a std::istream expression from a bool function, which C++11 and
// later reject, and it needs boost::tokenizer. This stand-in keeps the class
// name and its typed lookups (GetArgument) over a "Key=Value;Key=Value" map,
// which is all the factories built here use.
#pragma once

#include <map>
#include <string>
#include <sstream>
#include <vector>

#include "System/IlluminaPRT.h"
#include "Exception/Exception.h"

namespace Illumina
{
	namespace Core
	{
		class ArgumentMap
		{
			std::map<std::string, std::string> m_argumentMap;

		public:
			ArgumentMap(void) { }
			ArgumentMap(const ArgumentMap &o) : m_argumentMap(o.m_argumentMap) { }
			ArgumentMap(const std::map<std::string, std::string> m) : m_argumentMap(m) { }
			ArgumentMap(const std::string &s) { Initialise(s); }

			void Initialise(const std::map<std::string, std::string> m) { m_argumentMap = m; }

			void Initialise(const std::string &s)
			{
				m_argumentMap.clear();
				std::vector<std::string> tok;
				std::string cur;
				for (size_t i = 0; i < s.size(); i++) {
					if (s[i] == '=' || s[i] == ';') { if (!cur.empty()) tok.push_back(cur); cur.clear(); }
					else cur += s[i];
				}
				if (!cur.empty()) tok.push_back(cur);
				if (tok.size() % 2) throw new Exception("Invalid argument string!");
				for (size_t i = 0; i + 1 < tok.size(); i += 2) m_argumentMap[tok[i]] = tok[i + 1];
			}

			bool ContainsArgument(const std::string &k) { return m_argumentMap.find(k) != m_argumentMap.end(); }

			template <class T>
			bool GetArgument(const std::string &k, T &v)
			{
				if (!ContainsArgument(k)) return false;
				std::stringstream s(m_argumentMap[k]);
				return (bool)(s >> v);
			}

			std::string ToString(void)
			{
				std::string out;
				for (std::map<std::string, std::string>::iterator it = m_argumentMap.begin(); it != m_argumentMap.end(); ++it)
					out += it->first + "=" + it->second + ";";
				return out;
			}
		};
	}
}
