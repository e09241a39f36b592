// Minimal JSON reader and writer for checkpoint metadata (objects, arrays, strings, numbers,
// booleans, null). Enough for the UniformCUDA checkpoint format; not a general library.
#pragma once

#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace fc::json
{

struct Value
{
    enum Kind
    {
        Null,
        Bool,
        Number,
        String,
        Array,
        Object
    } kind = Null;
    bool boolean = false;
    double number = 0.0;
    std::string text;
    std::vector<Value> items;
    std::map<std::string, Value> fields;

    const Value* find(const std::string& key) const
    {
        const auto it = fields.find(key);
        return it == fields.end() ? nullptr : &it->second;
    }
};

class Parser
{
public:
    explicit Parser(const std::string& source) : s(source) {}

    Value parse()
    {
        Value v = value();
        space();
        if (pos != s.size())
            throw std::runtime_error("trailing characters in JSON");
        return v;
    }

private:
    const std::string& s;
    size_t pos = 0;

    void space()
    {
        while (pos < s.size() && (s[pos] == ' ' || s[pos] == '\n' || s[pos] == '\r' || s[pos] == '\t'))
            ++pos;
    }

    bool take(char c)
    {
        space();
        if (pos < s.size() && s[pos] == c)
        {
            ++pos;
            return true;
        }
        return false;
    }

    void expect(char c)
    {
        if (!take(c))
            throw std::runtime_error(std::string("expected '") + c + "' in JSON");
    }

    std::string string_body()
    {
        std::string out;
        while (pos < s.size() && s[pos] != '"')
        {
            char c = s[pos++];
            if (c == '\\')
            {
                if (pos >= s.size())
                    break;
                const char e = s[pos++];
                switch (e)
                {
                case 'n': out += '\n'; break;
                case 't': out += '\t'; break;
                case 'r': out += '\r'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'u':
                    if (pos + 4 > s.size())
                        throw std::runtime_error("bad escape in JSON");
                    out += '?';
                    pos += 4;
                    break;
                default: out += e; break;
                }
            }
            else
                out += c;
        }
        if (pos >= s.size())
            throw std::runtime_error("unterminated JSON string");
        ++pos;
        return out;
    }

    Value value()
    {
        space();
        if (pos >= s.size())
            throw std::runtime_error("unexpected end of JSON");
        Value v;
        const char c = s[pos];
        if (c == '{')
        {
            ++pos;
            v.kind = Value::Object;
            if (take('}'))
                return v;
            do
            {
                expect('"');
                const std::string key = string_body();
                expect(':');
                v.fields[key] = value();
            } while (take(','));
            expect('}');
        }
        else if (c == '[')
        {
            ++pos;
            v.kind = Value::Array;
            if (take(']'))
                return v;
            do
                v.items.push_back(value());
            while (take(','));
            expect(']');
        }
        else if (c == '"')
        {
            ++pos;
            v.kind = Value::String;
            v.text = string_body();
        }
        else if (s.compare(pos, 4, "true") == 0)
        {
            pos += 4;
            v.kind = Value::Bool;
            v.boolean = true;
        }
        else if (s.compare(pos, 5, "false") == 0)
        {
            pos += 5;
            v.kind = Value::Bool;
        }
        else if (s.compare(pos, 4, "null") == 0)
            pos += 4;
        else
        {
            size_t used = 0;
            v.kind = Value::Number;
            v.number = std::stod(s.substr(pos, 40), &used);
            if (used == 0)
                throw std::runtime_error("bad JSON number");
            pos += used;
        }
        return v;
    }
};

inline std::string number(double v)
{
    if (!std::isfinite(v))
        return "null";
    char buffer[40];
    std::snprintf(buffer, sizeof(buffer), "%.17g", v);
    return buffer;
}

inline std::string quoted(const std::string& v)
{
    std::string out = "\"";
    for (char c : v)
    {
        if (c == '"' || c == '\\')
            out += '\\';
        out += c;
    }
    return out + "\"";
}

} // namespace fc::json
