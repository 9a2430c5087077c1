// Minimal INI reader with the lookup rules the reference relies on
// (common/inih/INIReader.h as used by common/src/arguments.cpp:69-133):
// [section] headers, `key = value` lines, `;`/`#` full-line comments and `;`
// inline comments, case-insensitive section and key names, integers via
// strtol, booleans true/yes/on/1 and false/no/off/0.
#pragma once
#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <map>
#include <string>

class IniFile {
public:
    bool load(const std::string& path)
    {
        std::ifstream in(path);
        if (!in) return false;
        std::string line, section;
        while (std::getline(in, line)) {
            std::string s = trim(line);
            if (s.empty() || s[0] == ';' || s[0] == '#') continue;
            if (s[0] == '[') {
                size_t e = s.find(']');
                if (e != std::string::npos) section = lower(trim(s.substr(1, e - 1)));
                continue;
            }
            size_t eq = s.find_first_of("=:");
            if (eq == std::string::npos) continue;
            std::string key = lower(trim(s.substr(0, eq)));
            std::string val = s.substr(eq + 1);
            size_t c = val.find(';');
            if (c != std::string::npos) val = val.substr(0, c);
            values_[section + "=" + key] = trim(val);
        }
        return true;
    }
    std::string get(const std::string& sec, const std::string& key, const std::string& def) const
    {
        auto it = values_.find(lower(sec) + "=" + lower(key));
        return it == values_.end() ? def : it->second;
    }
    long get_int(const std::string& sec, const std::string& key, long def) const
    {
        std::string v = get(sec, key, "");
        if (v.empty()) return def;
        char* end = nullptr;
        long r = strtol(v.c_str(), &end, 0);
        return (end && end != v.c_str()) ? r : def;
    }
    bool get_bool(const std::string& sec, const std::string& key, bool def) const
    {
        std::string v = lower(get(sec, key, ""));
        if (v == "true" || v == "yes" || v == "on" || v == "1") return true;
        if (v == "false" || v == "no" || v == "off" || v == "0") return false;
        return def;
    }

private:
    std::map<std::string, std::string> values_;
    static std::string trim(const std::string& s)
    {
        size_t a = 0, b = s.size();
        while (a < b && isspace((unsigned char)s[a])) a++;
        while (b > a && isspace((unsigned char)s[b - 1])) b--;
        return s.substr(a, b - a);
    }
    static std::string lower(std::string s)
    {
        std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)tolower(c); });
        return s;
    }
};
