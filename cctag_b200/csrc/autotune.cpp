// JSON cache of cctagb_autotune's choices: a small reader for the file's
// subset of JSON (objects, arrays, strings, numbers, literals) and a writer
// that replaces the file through a temporary file and a rename.
#include "autotune.hpp"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <vector>

#include <unistd.h>

#include "common.hpp"

namespace cctagb {
namespace tune {

namespace {

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    double num = 0;
    bool b = false;
    std::string str;
    std::vector<Value> arr;
    std::map<std::string, Value> obj;
};

class Reader {
public:
    explicit Reader(const std::string& s) : s_(s) {}
    bool parse(Value& v)
    {
        if (!value(v, 0)) return false;
        ws();
        return i_ == s_.size();
    }

private:
    static constexpr int kMaxDepth = 32;
    const std::string& s_;
    size_t i_ = 0;

    void ws()
    {
        while (i_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[i_]))) ++i_;
    }
    bool lit(const char* w)
    {
        const size_t n = std::char_traits<char>::length(w);
        if (s_.compare(i_, n, w) != 0) return false;
        i_ += n;
        return true;
    }
    bool string(std::string& out)
    {
        if (i_ >= s_.size() || s_[i_] != '"') return false;
        ++i_;
        out.clear();
        while (i_ < s_.size()) {
            const char c = s_[i_++];
            if (c == '"') return true;
            if (static_cast<unsigned char>(c) < 0x20) return false;
            if (c != '\\') {
                out.push_back(c);
                continue;
            }
            if (i_ >= s_.size()) return false;
            const char e = s_[i_++];
            switch (e) {
                case '"': out.push_back('"'); break;
                case '\\': out.push_back('\\'); break;
                case '/': out.push_back('/'); break;
                case 'b': out.push_back('\b'); break;
                case 'f': out.push_back('\f'); break;
                case 'n': out.push_back('\n'); break;
                case 'r': out.push_back('\r'); break;
                case 't': out.push_back('\t'); break;
                case 'u': {  // keys are ASCII: other code points become '?'
                    if (i_ + 4 > s_.size()) return false;
                    unsigned cp = 0;
                    for (int k = 0; k < 4; ++k) {
                        const char h = s_[i_++];
                        if (!std::isxdigit(static_cast<unsigned char>(h))) return false;
                        cp = cp * 16 + unsigned(std::isdigit(static_cast<unsigned char>(h)) ? h - '0'
                                                                                          : (std::tolower(h) - 'a' + 10));
                    }
                    out.push_back(cp < 0x80 ? char(cp) : '?');
                    break;
                }
                default: return false;
            }
        }
        return false;
    }
    bool number(double& out)
    {
        const char* b = s_.c_str() + i_;
        char* e = nullptr;
        out = std::strtod(b, &e);
        if (e == b) return false;
        i_ += size_t(e - b);
        return true;
    }
    bool value(Value& v, int depth)
    {
        if (depth > kMaxDepth) return false;
        ws();
        if (i_ >= s_.size()) return false;
        const char c = s_[i_];
        if (c == '{') {
            ++i_;
            v.kind = Value::Object;
            ws();
            if (i_ < s_.size() && s_[i_] == '}') {
                ++i_;
                return true;
            }
            for (;;) {
                ws();
                std::string k;
                if (!string(k)) return false;
                ws();
                if (i_ >= s_.size() || s_[i_] != ':') return false;
                ++i_;
                Value item;
                if (!value(item, depth + 1)) return false;
                v.obj[k] = std::move(item);
                ws();
                if (i_ < s_.size() && s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (i_ < s_.size() && s_[i_] == '}') {
                    ++i_;
                    return true;
                }
                return false;
            }
        }
        if (c == '[') {
            ++i_;
            v.kind = Value::Array;
            ws();
            if (i_ < s_.size() && s_[i_] == ']') {
                ++i_;
                return true;
            }
            for (;;) {
                Value item;
                if (!value(item, depth + 1)) return false;
                v.arr.push_back(std::move(item));
                ws();
                if (i_ < s_.size() && s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (i_ < s_.size() && s_[i_] == ']') {
                    ++i_;
                    return true;
                }
                return false;
            }
        }
        if (c == '"') {
            v.kind = Value::String;
            return string(v.str);
        }
        if (lit("true")) {
            v.kind = Value::Bool;
            v.b = true;
            return true;
        }
        if (lit("false")) {
            v.kind = Value::Bool;
            return true;
        }
        if (lit("null")) return true;
        v.kind = Value::Number;
        return number(v.num);
    }
};

std::string quoted(const std::string& s)
{
    std::string o = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') {
            o.push_back('\\');
            o.push_back(c);
        } else if (static_cast<unsigned char>(c) < 0x20) {
            char buf[8];
            std::snprintf(buf, sizeof(buf), "\\u%04x", unsigned(static_cast<unsigned char>(c)));
            o += buf;
        } else {
            o.push_back(c);
        }
    }
    return o + "\"";
}

bool read_file(const std::string& path, std::string& out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

// The entries of a cache file of this version; false when the file is absent,
// malformed or of another version.
bool read_entries(const std::string& path, std::map<std::string, Value>& entries)
{
    std::string text;
    if (!read_file(path, text)) return false;
    Value root;
    if (!Reader(text).parse(root) || root.kind != Value::Object) return false;
    auto v = root.obj.find("version");
    if (v == root.obj.end() || v->second.kind != Value::Number || v->second.num != double(kCacheVersion)) return false;
    auto e = root.obj.find("entries");
    if (e == root.obj.end() || e->second.kind != Value::Object) return false;
    entries = e->second.obj;
    return true;
}

bool int_field(const Value& o, const char* name, int lo, int hi, int& out)
{
    auto it = o.obj.find(name);
    if (it == o.obj.end() || it->second.kind != Value::Number) return false;
    const double d = it->second.num;
    if (!(d >= lo && d <= hi) || d != double(int(d))) return false;
    out = int(d);
    return true;
}

}  // namespace

namespace {

std::string key_of(const char* gpu_name, int sm_count, const std::string& size, int frames, int n_crowns)
{
    std::string g = gpu_name ? gpu_name : "";
    for (char& c : g)
        if (c == '|' || c == '"' || c == '\\' || static_cast<unsigned char>(c) < 0x20) c = '_';
    return g + "|sm" + std::to_string(sm_count) + "|" + size + "|f" + std::to_string(frames) + "|c" +
           std::to_string(n_crowns);
}

}  // namespace

std::string key(const char* gpu_name, int sm_count, int w, int h, int frames, int n_crowns)
{
    return key_of(gpu_name, sm_count, std::to_string(w) + "x" + std::to_string(h), frames, n_crowns);
}

std::string key_mixed(const char* gpu_name, int sm_count, long long total_px, int frames, int n_crowns)
{
    return key_of(gpu_name, sm_count, "mixed" + std::to_string(total_px), frames, n_crowns);
}

bool cache_get(const std::string& path, const std::string& k, cctagb_tune_choice& out)
{
    std::map<std::string, Value> entries;
    if (!read_entries(path, entries)) return false;
    auto it = entries.find(k);
    if (it == entries.end() || it->second.kind != Value::Object) return false;
    cctagb_tune_choice c{};
    if (!int_field(it->second, "batchWaveFrames", 1, kMaxBatchFrames, c.batchWaveFrames)) return false;
    if (!int_field(it->second, "identLayout", CCTAGB_IDENT_AUTO, CCTAGB_IDENT_BLOCK, c.identLayout)) return false;
    if (!int_field(it->second, "hostThreads", 0, 64, c.hostThreads)) return false;
    auto ms = it->second.obj.find("ms_per_frame");
    if (ms != it->second.obj.end() && ms->second.kind == Value::Number) c.ms_per_frame = float(ms->second.num);
    c.from_cache = 1;
    out = c;
    return true;
}

void cache_put(const std::string& path, const std::string& k, const cctagb_tune_choice& c)
{
    std::map<std::string, Value> entries;
    read_entries(path, entries);  // an absent or unreadable file starts empty
    Value e;
    e.kind = Value::Object;
    auto num = [](double d) {
        Value v;
        v.kind = Value::Number;
        v.num = d;
        return v;
    };
    e.obj["batchWaveFrames"] = num(c.batchWaveFrames);
    e.obj["identLayout"] = num(c.identLayout);
    e.obj["hostThreads"] = num(c.hostThreads);
    e.obj["ms_per_frame"] = num(c.ms_per_frame);
    entries[k] = e;
    std::ostringstream o;
    o << "{\n  \"version\": " << kCacheVersion << ",\n  \"entries\": {";
    bool first = true;
    for (const auto& kv : entries) {
        if (kv.second.kind != Value::Object) continue;
        o << (first ? "\n" : ",\n") << "    " << quoted(kv.first) << ": {";
        bool f2 = true;
        for (const auto& f : kv.second.obj) {
            if (f.second.kind != Value::Number) continue;
            char buf[64];
            std::snprintf(buf, sizeof(buf), "%.9g", f.second.num);
            o << (f2 ? "" : ", ") << quoted(f.first) << ": " << buf;
            f2 = false;
        }
        o << "}";
        first = false;
    }
    o << "\n  }\n}\n";
    const std::string tmp = path + ".tmp." + std::to_string(long(::getpid()));
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        if (!f) throw Error{CCTAGB_BAD_ARG, "cannot write the tuning cache " + tmp};
        f << o.str();
        if (!f.good()) throw Error{CCTAGB_BAD_ARG, "cannot write the tuning cache " + tmp};
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        throw Error{CCTAGB_BAD_ARG, "cannot replace the tuning cache " + path};
    }
}

}  // namespace tune
}  // namespace cctagb
