// Replacement for the reference's System/ArgumentMap.h, found first on the
// include path when the engine headers are compiled here (the GPU space plug-in
// and the CPU checker built from the reference sources).
//
// Why: the reference's ArgumentMap (Core/System/ArgumentMap.h:243-258)
// returns a std::istream expression from a bool function, which C++11 and
// later reject, and it needs boost::tokenizer. This stand-in keeps the class
// name and its typed lookups (GetArgument) over a "Key=Value;Key=Value" map.
// Brace lists keep the reference's text forms: "{a,b,c}" for Vector2/3,
// Spectrum and RGBPixel, "{{a,b,c},{d,e,f}}" for lists of them,
// "{a,b,...,i}" for a row-major Matrix3x3 and "{x,y,z}" for a list of names
// (Core/System/ArgumentMap.h:99-262); numbers are read as floats.
#pragma once

#include <map>
#include <string>
#include <sstream>
#include <vector>

#include "System/IlluminaPRT.h"
#include "Exception/Exception.h"
#include "Geometry/Matrix3x3.h"
#include "Geometry/Vector2.h"
#include "Geometry/Vector3.h"
#include "Image/RGBPixel.h"
#include "Spectrum/Spectrum.h"

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

			// A brace list as its items: the text between separators '{', ','
			// and '}', with empty items dropped.
			static std::vector<std::string> Items(const std::string &s)
			{
				std::vector<std::string> out;
				std::string cur;
				for (size_t i = 0; i < s.size(); i++) {
					if (s[i] == '{' || s[i] == '}' || s[i] == ',') { if (!cur.empty()) out.push_back(cur); cur.clear(); }
					else cur += s[i];
				}
				if (!cur.empty()) out.push_back(cur);
				return out;
			}

			// Every number of a brace list, in order; false if an item is not one.
			bool Numbers(const std::string &k, std::vector<float> &out)
			{
				if (!ContainsArgument(k)) return false;
				std::vector<std::string> items = Items(m_argumentMap[k]);
				out.clear();
				for (size_t i = 0; i < items.size(); i++) {
					std::stringstream s(items[i]);
					float f;
					if (!(s >> f)) return false;
					out.push_back(f);
				}
				return true;
			}

			bool GetArgument(const std::string &k, std::vector<std::string> &v)
			{
				if (!ContainsArgument(k)) return false;
				std::vector<std::string> items = Items(m_argumentMap[k]);
				v.insert(v.end(), items.begin(), items.end());
				return true;
			}

			bool GetArgument(const std::string &k, Vector2 &v)
			{
				std::vector<float> f;
				if (!Numbers(k, f) || f.size() < 2) return false;
				v = Vector2(f[0], f[1]);
				return true;
			}

			bool GetArgument(const std::string &k, Vector3 &v)
			{
				std::vector<float> f;
				if (!Numbers(k, f) || f.size() < 3) return false;
				v = Vector3(f[0], f[1], f[2]);
				return true;
			}

			bool GetArgument(const std::string &k, std::vector<Vector3> &v)
			{
				std::vector<float> f;
				if (!Numbers(k, f)) return false;
				for (size_t i = 0; i + 2 < f.size(); i += 3) v.push_back(Vector3(f[i], f[i + 1], f[i + 2]));
				return true;
			}

			bool GetArgument(const std::string &k, RGBPixel &v)
			{
				std::vector<float> f;
				if (!Numbers(k, f) || f.size() < 3) return false;
				v.Set(f[0], f[1], f[2]);
				return true;
			}

			bool GetArgument(const std::string &k, Spectrum &v)
			{
				std::vector<float> f;
				if (!Numbers(k, f) || f.size() < 3) return false;
				v = Spectrum(f[0], f[1], f[2]);
				return true;
			}

			bool GetArgument(const std::string &k, std::vector<Spectrum> &v)
			{
				std::vector<float> f;
				if (!Numbers(k, f)) return false;
				for (size_t i = 0; i + 2 < f.size(); i += 3) v.push_back(Spectrum(f[i], f[i + 1], f[i + 2]));
				return true;
			}

			bool GetArgument(const std::string &k, Matrix3x3 &v)
			{
				std::vector<float> f;
				if (!Numbers(k, f) || f.size() < 9) return false;
				v._00 = f[0]; v._01 = f[1]; v._02 = f[2];
				v._10 = f[3]; v._11 = f[4]; v._12 = f[5];
				v._20 = f[6]; v._21 = f[7]; v._22 = f[8];
				return true;
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
