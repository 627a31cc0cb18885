// Minimal JSON reader for the circuit transport (the serde_json input of
// src/monolithic/statevector/simulator.rs:204-211).  Numbers keep the
// integer/float distinction serde relies on: a usize field accepts only a
// non-negative integer literal that fits in 64 bits, an f64 field accepts any
// number.  NaN/Infinity literals, trailing characters and nesting deeper than
// serde_json's limit of 128 are errors, as in serde_json.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace dq::json {

enum class Type { Null, Bool, Int, Float, String, Array, Object };

struct Value {
    Type type = Type::Null;
    bool b = false;
    bool negative = false;   // Int: sign
    bool int_overflow = false;  // Int literal beyond 64 bits (parsed as float by serde_json)
    uint64_t u = 0;          // Int: magnitude
    double f = 0.0;          // Int/Float: value as double
    std::string s;
    std::vector<Value> arr;
    std::vector<std::pair<std::string, Value>> obj;

    const Value* find(const std::string& key) const {
        const Value* hit = nullptr;
        for (auto& kv : obj)
            if (kv.first == key) hit = &kv.second;
        return hit;
    }
    int count(const std::string& key) const {
        int c = 0;
        for (auto& kv : obj)
            if (kv.first == key) c++;
        return c;
    }
};

// Throws std::runtime_error with a position-annotated message.
Value parse(const char* text, size_t len);

}  // namespace dq::json
