// Minimal JSON reader for the reference's input files (params.json,
// station.json).
//
// Semantics follow the reference's vendored cJSON where they affect values:
//  * object member lookup is case-insensitive and returns the first match
//    (src/cjson.c:793-799, cJSON_GetObjectItem with cJSON_strcasecmp), so
//    "out" satisfies a lookup of "OUT";
//  * numbers are parsed by accumulating decimal digits in a double and then
//    scaling by pow(10, exponent) (src/cjson.c:107-145), not by strtod; the
//    integer view of a number is the C cast (int)value.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace cgfdm {

struct JsonValue {
    enum Kind { Null, False, True, Number, String, Array, Object } kind = Null;
    double num = 0.0;
    std::string str;
    std::vector<JsonValue> items;                               // Array
    std::vector<std::pair<std::string, JsonValue>> members;     // Object, in file order

    int as_int() const { return (int)num; }
    // First member whose name matches case-insensitively, or nullptr.
    const JsonValue *get(const char *key) const;
};

// Parses text; on error returns false and sets err.
bool json_parse(const std::string &text, JsonValue &out, std::string &err);
bool json_parse_file(const std::string &path, JsonValue &out, std::string &err);

}  // namespace cgfdm
