// toml_lite.h -- the subset of TOML used by DG-MPI input decks: [Section]
// headers, `key = value` with strings, numbers, booleans and flat arrays,
// and # comments.  (The reference uses toml11, src/exec/main.cpp:38.)
#pragma once
#include <algorithm>
#include <cctype>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace dgh {

struct TomlValue {
    enum Kind { kString, kNumber, kBool, kArray } kind = kString;
    std::string s;
    double num = 0.0;
    bool b = false;
    std::vector<TomlValue> arr;
};

class Toml {
public:
    static Toml parse_file(const std::string& path)
    {
        std::ifstream f(path);
        if (!f) throw std::runtime_error("cannot open input deck " + path);
        std::stringstream ss;
        ss << f.rdbuf();
        return parse(ss.str());
    }

    static Toml parse(const std::string& text)
    {
        Toml t;
        std::string section;
        std::istringstream in(text);
        std::string line;
        int lineno = 0;
        while (std::getline(in, line)) {
            ++lineno;
            const std::string l = trim(strip_comment(line));
            if (l.empty()) continue;
            if (l.front() == '[') {
                if (l.back() != ']') throw std::runtime_error("bad section header at line " + std::to_string(lineno));
                section = trim(l.substr(1, l.size() - 2));
                continue;
            }
            const size_t eq = l.find('=');
            if (eq == std::string::npos) throw std::runtime_error("expected key = value at line " + std::to_string(lineno));
            const std::string key = trim(l.substr(0, eq));
            size_t pos = 0;
            const std::string rhs = trim(l.substr(eq + 1));
            t.values_[section + "." + key] = parse_value(rhs, pos, lineno);
        }
        return t;
    }

    bool has(const std::string& sec, const std::string& key) const { return values_.count(sec + "." + key) > 0; }

    const TomlValue& at(const std::string& sec, const std::string& key) const
    {
        auto it = values_.find(sec + "." + key);
        if (it == values_.end()) throw std::runtime_error("missing [" + sec + "] " + key);
        return it->second;
    }

    std::string str(const std::string& sec, const std::string& key) const
    {
        const TomlValue& v = at(sec, key);
        if (v.kind != TomlValue::kString) throw std::runtime_error("[" + sec + "] " + key + " must be a string");
        return v.s;
    }
    std::string str_or(const std::string& sec, const std::string& key, const std::string& d) const
    {
        return has(sec, key) ? str(sec, key) : d;
    }
    double num(const std::string& sec, const std::string& key) const
    {
        const TomlValue& v = at(sec, key);
        if (v.kind != TomlValue::kNumber) throw std::runtime_error("[" + sec + "] " + key + " must be a number");
        return v.num;
    }
    double num_or(const std::string& sec, const std::string& key, double d) const { return has(sec, key) ? num(sec, key) : d; }
    bool boolean(const std::string& sec, const std::string& key) const
    {
        const TomlValue& v = at(sec, key);
        if (v.kind != TomlValue::kBool) throw std::runtime_error("[" + sec + "] " + key + " must be true or false");
        return v.b;
    }
    std::vector<double> nums(const std::string& sec, const std::string& key) const
    {
        const TomlValue& v = at(sec, key);
        if (v.kind != TomlValue::kArray) throw std::runtime_error("[" + sec + "] " + key + " must be an array");
        std::vector<double> out;
        for (const auto& e : v.arr) {
            if (e.kind != TomlValue::kNumber) throw std::runtime_error("[" + sec + "] " + key + " must hold numbers");
            out.push_back(e.num);
        }
        return out;
    }

private:
    std::map<std::string, TomlValue> values_;

    static std::string strip_comment(const std::string& s)
    {
        bool in_str = false;
        for (size_t i = 0; i < s.size(); ++i) {
            if (s[i] == '"') in_str = !in_str;
            if (s[i] == '#' && !in_str) return s.substr(0, i);
        }
        return s;
    }
    static std::string trim(const std::string& s)
    {
        size_t a = 0, b = s.size();
        while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
        while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
        return s.substr(a, b - a);
    }
    static TomlValue parse_value(const std::string& s, size_t& pos, int lineno)
    {
        while (pos < s.size() && std::isspace(static_cast<unsigned char>(s[pos]))) ++pos;
        if (pos >= s.size()) throw std::runtime_error("missing value at line " + std::to_string(lineno));
        TomlValue v;
        if (s[pos] == '"') {
            const size_t end = s.find('"', pos + 1);
            if (end == std::string::npos) throw std::runtime_error("unterminated string at line " + std::to_string(lineno));
            v.kind = TomlValue::kString;
            v.s = s.substr(pos + 1, end - pos - 1);
            pos = end + 1;
        } else if (s[pos] == '[') {
            v.kind = TomlValue::kArray;
            ++pos;
            while (true) {
                while (pos < s.size() && (std::isspace(static_cast<unsigned char>(s[pos])) || s[pos] == ',')) ++pos;
                if (pos >= s.size()) throw std::runtime_error("unterminated array at line " + std::to_string(lineno));
                if (s[pos] == ']') { ++pos; break; }
                v.arr.push_back(parse_value(s, pos, lineno));
            }
        } else if (s.compare(pos, 4, "true") == 0 || s.compare(pos, 5, "false") == 0) {
            v.kind = TomlValue::kBool;
            v.b = s[pos] == 't';
            pos += v.b ? 4 : 5;
        } else {
            size_t end = pos;
            while (end < s.size() && (std::isalnum(static_cast<unsigned char>(s[end])) || s[end] == '.' || s[end] == '-' ||
                                      s[end] == '+' || s[end] == '_'))
                ++end;
            std::string tok = s.substr(pos, end - pos);
            tok.erase(std::remove(tok.begin(), tok.end(), '_'), tok.end());
            try {
                size_t used = 0;
                v.num = std::stod(tok, &used);
                if (used != tok.size()) throw std::invalid_argument(tok);
            } catch (const std::exception&) {
                throw std::runtime_error("bad number '" + tok + "' at line " + std::to_string(lineno));
            }
            v.kind = TomlValue::kNumber;
            pos = end;
        }
        return v;
    }
};

}  // namespace dgh
