// Stand-in for <bitloop/util/json.h>. bitloop's JSON type follows nlohmann::json; when that
// header is on the include path the stand-in is exactly it, otherwise a minimal holder that is
// enough for the code that only stores checkpoint metadata.
#pragma once
#if __has_include(<nlohmann/json.hpp>)
#include <nlohmann/json.hpp>
namespace bl::JSON
{
using json = nlohmann::json;
}
#else
#include <map>
#include <string>

namespace bl::JSON
{
struct json
{
    std::map<std::string, std::string> fields;
};
}
#endif
