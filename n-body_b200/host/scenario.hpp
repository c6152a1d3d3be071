// Scenario I/O of the host layer: the reference's JSON scenario schema and its tipsy reader.
//
//   JSON  NBody::to_json / from_json (src/NBody/Simulation/Simulation.cpp:154-228): an object with
//         "particles": [ { "position": {x, y, z}, "velocity": {x, y, z}, "mass": m,
//         "acceleration": {x, y, z}, ... } ], plus an optional top-level "G" that sets the rule's
//         constant (src/Application/Application.cpp:147-152). Particles are written in particle
//         order; unknown keys (colour, sphere radius) are ignored on input and not written.
//   tipsy NBody::from_tipsy (Simulation.cpp:273-395): 28-byte header (double time; uint32 n,
//         ndim, ngas, ndark, nstar), big- or little-endian (decided by ndim in 1..3), an optional
//         4-byte pad (decided by the file size); gas particles are read only when there are no
//         stars, dark matter is skipped, stars are read. Each particle: mass, position, velocity,
//         then 5 (gas) or 4 (star) more floats that are not used.
#pragma once

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "nbody_b200.hpp"

namespace nbody_b200 {

// A small JSON value and parser (objects, arrays, numbers, strings, booleans, null).
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    const Json *find(const std::string &k) const {
        for (auto &kv: obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

class JsonParser {
public:
    explicit JsonParser(const std::string &text) : s(text) {}

    Json parse() {
        Json v = value();
        ws();
        if (i != s.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string &s;
    std::size_t i = 0;

    [[noreturn]] void fail(const char *what) {
        throw Error(NB_ERR_INVALID_ARGUMENT, std::string("JSON: ") + what + " at offset " + std::to_string(i));
    }
    void ws() {
        while (i < s.size() && std::isspace((unsigned char) s[i])) ++i;
    }
    bool lit(const char *w) {
        const std::size_t n = std::strlen(w);
        if (s.compare(i, n, w) == 0) {
            i += n;
            return true;
        }
        return false;
    }
    Json value() {
        ws();
        if (i >= s.size()) fail("unexpected end");
        Json v;
        const char c = s[i];
        if (c == '{') {
            v.kind = Json::Object;
            ++i;
            ws();
            if (i < s.size() && s[i] == '}') {
                ++i;
                return v;
            }
            for (;;) {
                ws();
                if (i >= s.size() || s[i] != '"') fail("expected a key");
                std::string k = string();
                ws();
                if (i >= s.size() || s[i] != ':') fail("expected ':'");
                ++i;
                v.obj.emplace_back(std::move(k), value());
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == '}') { ++i; return v; }
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = Json::Array;
            ++i;
            ws();
            if (i < s.size() && s[i] == ']') {
                ++i;
                return v;
            }
            for (;;) {
                v.arr.push_back(value());
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == ']') { ++i; return v; }
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = Json::String;
            v.str = string();
            return v;
        }
        if (lit("true")) { v.kind = Json::Bool; v.b = true; return v; }
        if (lit("false")) { v.kind = Json::Bool; v.b = false; return v; }
        if (lit("null")) return v;
        const char *begin = s.c_str() + i;
        char *end = nullptr;
        v.num = std::strtod(begin, &end);
        if (end == begin) fail("unexpected character");
        i += (std::size_t) (end - begin);
        v.kind = Json::Number;
        return v;
    }
    std::string string() {
        std::string out;
        ++i;  // opening quote
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\') {
                ++i;
                if (i >= s.size()) fail("bad escape");
                const char e = s[i];
                if (e == 'u') {
                    if (i + 4 >= s.size()) fail("bad escape");
                    i += 4;  // code points are not needed by the schema; keep a placeholder
                    out.push_back('?');
                } else {
                    out.push_back(e == 'n' ? '\n' : e == 't' ? '\t' : e == 'r' ? '\r' : e == 'b' ? '\b'
                                  : e == 'f' ? '\f' : e);
                }
                ++i;
            } else {
                out.push_back(s[i++]);
            }
        }
        if (i >= s.size()) fail("unterminated string");
        ++i;
        return out;
    }
};

struct Scenario {
    Simulation simulation;
    bool hasG = false;
    float G = 1.0f;
};

inline vec3 json_vec3(const Json &j) {
    auto comp = [&](const char *k) {
        const Json *c = j.find(k);
        if (!c || c->kind != Json::Number) throw Error(NB_ERR_INVALID_ARGUMENT, std::string("JSON: vector lacks ") + k);
        return (float) c->num;
    };
    return {comp("x"), comp("y"), comp("z")};
}

// NBody::from_json (Simulation.cpp:187-228)
inline Scenario scenario_from_json(const std::string &text) {
    Json root = JsonParser(text).parse();
    if (root.kind != Json::Object) throw Error(NB_ERR_INVALID_ARGUMENT, "JSON: top level is not an object");
    Scenario sc;
    if (const Json *g = root.find("G")) {
        sc.hasG = true;
        sc.G = (float) g->num;
    }
    const Json *ps = root.find("particles");
    if (!ps || ps->kind != Json::Array) throw Error(NB_ERR_INVALID_ARGUMENT, "JSON: no \"particles\" array");
    for (const Json &p: ps->arr) {
        vec3 pos, vel;
        float m = 0.f;
        if (const Json *v = p.find("position")) pos = json_vec3(*v);
        if (const Json *v = p.find("velocity")) vel = json_vec3(*v);
        if (const Json *v = p.find("mass")) m = (float) v->num;
        const std::size_t k = sc.simulation.newParticle(pos, vel, m);
        if (const Json *v = p.find("acceleration")) sc.simulation.acceleration[k] = json_vec3(*v);
    }
    return sc;
}

inline std::string float_text(float v) {
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%.9g", (double) v);
    return buf;
}

// NBody::to_json (Simulation.cpp:154-185): particles in particle order.
inline std::string scenario_to_json(const Simulation &s, const float *G = nullptr) {
    std::ostringstream o;
    o << "{\n";
    if (G) o << "    \"G\": " << float_text(*G) << ",\n";
    o << "    \"particles\": [";
    auto v3 = [&](const vec3 &v) {
        return "{\"x\": " + float_text(v.x) + ", \"y\": " + float_text(v.y) + ", \"z\": " + float_text(v.z) + "}";
    };
    for (std::size_t i = 0; i < s.particleCount(); ++i) {
        o << (i ? ",\n        " : "\n        ");
        o << "{\"position\": " << v3(s.position[i]) << ", \"velocity\": " << v3(s.velocity[i])
          << ", \"mass\": " << float_text(s.mass[i]) << ", \"acceleration\": " << v3(s.acceleration[i]) << "}";
    }
    o << "\n    ]\n}\n";
    return o.str();
}

template<typename T>
inline T tipsy_swap(T v, bool swap) {
    if (!swap) return v;
    unsigned char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    for (std::size_t k = 0; k < sizeof(T) / 2; ++k) std::swap(b[k], b[sizeof(T) - 1 - k]);
    std::memcpy(&v, b, sizeof(T));
    return v;
}

// NBody::from_tipsy (Simulation.cpp:273-395)
inline Scenario scenario_from_tipsy(const std::string &path) {
    std::ifstream in(path, std::ios::binary);
    if (!in.good()) throw Error(NB_ERR_INVALID_ARGUMENT, "cannot open " + path);
    in.seekg(0, std::ios::end);
    const uint64_t fs = (uint64_t) in.tellg();
    in.seekg(0, std::ios::beg);
    double t = 0.0;
    uint32_t n = 0, ndim = 0, ng = 0, nd = 0, ns = 0;
    in.read(reinterpret_cast<char *>(&t), 8);
    in.read(reinterpret_cast<char *>(&n), 4);
    in.read(reinterpret_cast<char *>(&ndim), 4);
    in.read(reinterpret_cast<char *>(&ng), 4);
    in.read(reinterpret_cast<char *>(&nd), 4);
    in.read(reinterpret_cast<char *>(&ns), 4);
    if (!in.good()) throw Error(NB_ERR_INVALID_ARGUMENT, "tipsy: truncated header");
    const bool swap = (ndim < 1 || 3 < ndim);
    ng = tipsy_swap(ng, swap);
    nd = tipsy_swap(nd, swap);
    ns = tipsy_swap(ns, swap);
    const uint64_t body = 48ull * ng + 36ull * nd + 44ull * ns;
    if (fs == 32 + body) in.seekg(4, std::ios::cur);
    else if (fs != 28 + body) throw Error(NB_ERR_INVALID_ARGUMENT, "tipsy: file size does not match header");
    Scenario sc;
    auto rd = [&]() {
        float v = 0.f;
        in.read(reinterpret_cast<char *>(&v), 4);
        return tipsy_swap(v, swap);
    };
    auto particle = [&](int extra) {
        const float m = rd();
        const vec3 p{rd(), rd(), rd()};
        const vec3 v{rd(), rd(), rd()};
        for (int k = 0; k < extra; ++k) rd();
        sc.simulation.newParticle(p, v, m);
    };
    if (ns > 0) in.seekg(48ll * ng, std::ios::cur);  // gas is read only without stars
    else
        for (uint32_t k = 0; k < ng; ++k) particle(5);
    in.seekg(36ll * nd, std::ios::cur);  // dark matter is skipped
    for (uint32_t k = 0; k < ns; ++k) particle(4);
    if (!in.good()) throw Error(NB_ERR_INVALID_ARGUMENT, "tipsy: truncated particle data");
    return sc;
}

inline std::string read_text(const std::string &path) {
    std::ifstream in(path, std::ios::binary);
    if (!in.good()) throw Error(NB_ERR_INVALID_ARGUMENT, "cannot open " + path);
    std::ostringstream o;
    o << in.rdbuf();
    return o.str();
}

// A scenario file by extension: .json, else tipsy.
inline Scenario load_scenario(const std::string &path) {
    const std::size_t dot = path.find_last_of('.');
    const std::string ext = dot == std::string::npos ? "" : path.substr(dot);
    if (ext == ".json") return scenario_from_json(read_text(path));
    return scenario_from_tipsy(path);
}

}  // namespace nbody_b200
