// Stand-in for <bitloop/util/json.h>: the checkpoint metadata type only needs to exist.
#pragma once
#include <map>
#include <string>

namespace bl::JSON
{
struct json
{
    std::map<std::string, std::string> fields;
};
}
