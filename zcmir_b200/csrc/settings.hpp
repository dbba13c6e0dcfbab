// Engine settings: every key of the reference's Settings (src/settings.zig:38-178) with its
// default, applied from a JSON object (unknown keys and wrong types are errors) and dumped as
// one JSON object with enums as strings.
#pragma once

#include <string>
#include <vector>

namespace zc {

enum class Kind { Bool, U32, F64, Enum };

struct KeyDef {
    const char* name;
    Kind kind;
    const char* const* values;  // enum names (Kind::Enum), null-terminated
    double dnum;                // default of Bool / U32 / F64
    const char* dstr;           // default of Enum
};

class Settings {
  public:
    Settings();
    // Apply a JSON object of overrides; on error nothing changes and `err` says why.
    bool apply(const char* json, size_t len, std::string& err);
    std::string to_json() const;

    bool b(const char* key) const;
    double f(const char* key) const;
    unsigned u(const char* key) const;
    const std::string& e(const char* key) const;
    // for tests and the engine: set one key from a JSON value text
    static int index_of(const std::string& key);
    static int count();
    static const KeyDef& def(int i);

  private:
    std::vector<double> num_;
    std::vector<std::string> str_;
};

}  // namespace zc
