#include "dict.h"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "cfg_internal.h"

namespace cfg
{

namespace
{

bool isNumber(const std::string& s, double& v)
{
    if (s.empty()) return false;
    char* end = nullptr;
    v = std::strtod(s.c_str(), &end);
    return end == s.c_str() + s.size();
}

}  // namespace

struct DictParser
{
    const std::string& s;
    size_t i = 0;

    explicit DictParser(const std::string& src) : s(src) {}

    void skip()
    {
        for (;;)
        {
            while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
            if (i < s.size() && s[i] == '#')
            {
                while (i < s.size() && s[i] != '\n') ++i;
                continue;
            }
            if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/')
            {
                while (i < s.size() && s[i] != '\n') ++i;
                continue;
            }
            return;
        }
    }

    // a token: one of { } ; ( ) or a word / quoted string; empty at the end
    std::string token(bool& punct, bool& quoted)
    {
        skip();
        punct = quoted = false;
        if (i >= s.size()) return {};
        const char c = s[i];
        if (c == '{' || c == '}' || c == ';' || c == '(' || c == ')')
        {
            ++i;
            punct = true;
            return std::string(1, c);
        }
        if (c == '"')
        {
            ++i;
            std::string out;
            while (i < s.size() && s[i] != '"') out.push_back(s[i++]);
            if (i < s.size()) ++i;
            quoted = true;
            return out;
        }
        std::string out;
        while (i < s.size() && !std::isspace(static_cast<unsigned char>(s[i])) && s[i] != '{' && s[i] != '}' &&
               s[i] != ';' && s[i] != '(' && s[i] != ')')
            out.push_back(s[i++]);
        return out;
    }

    void parseBody(Dict& d, bool nested)
    {
        for (;;)
        {
            bool punct, quoted;
            const std::string key = token(punct, quoted);
            if (key.empty() && !punct && !quoted)
            {
                if (nested) fail(CFG_ESETUP, "dictionary: unexpected end inside a block");
                return;
            }
            if (punct && key == "}")
            {
                if (!nested) fail(CFG_ESETUP, "dictionary: unbalanced '}'");
                return;
            }
            if (punct && key == ";") continue;
            if (punct) fail(CFG_ESETUP, "dictionary: expected key, got '" + key + "'");
            Dict::Entry e;
            const std::string t = token(punct, quoted);
            if (punct && t == "{")
            {
                e.kind = Dict::Entry::Block;
                e.block = std::make_shared<Dict>();
                parseBody(*e.block, true);
            }
            else if (punct && t == "(")
            {
                e.kind = Dict::Entry::List;
                for (;;)
                {
                    const std::string it = token(punct, quoted);
                    if (punct && it == ")") break;
                    if (it.empty() && !quoted) fail(CFG_ESETUP, "dictionary: unterminated list for '" + key + "'");
                    e.items.push_back(it);
                }
                expectSemi(key);
            }
            else if (!punct && (!t.empty() || quoted))
            {
                double v;
                if (!quoted && isNumber(t, v))
                {
                    e.kind = Dict::Entry::Number;
                    e.number = v;
                }
                e.word = t;
                expectSemi(key);
            }
            else
            {
                fail(CFG_ESETUP, "dictionary: bad value for '" + key + "'");
            }
            if (!d.entries_.count(key)) d.order_.push_back(key);
            d.entries_[key] = std::move(e);
        }
    }

    void expectSemi(const std::string& key)
    {
        bool punct, quoted;
        const std::string t = token(punct, quoted);
        if (!(punct && t == ";")) fail(CFG_ESETUP, "dictionary: missing ';' after '" + key + "'");
    }
};

Dict Dict::parse(const std::string& text)
{
    Dict d;
    DictParser p(text);
    p.parseBody(d, false);
    return d;
}

Dict Dict::parseFile(const std::string& path)
{
    std::ifstream in(path);
    if (!in) fail(CFG_ESETUP, "dictionary: cannot open " + path);
    std::stringstream ss;
    ss << in.rdbuf();
    return parse(ss.str());
}

const Dict::Entry& Dict::get(const std::string& k) const
{
    auto it = entries_.find(k);
    if (it == entries_.end()) fail(CFG_ESETUP, "dictionary: missing key '" + k + "'");
    return it->second;
}

const Dict& Dict::dict(const std::string& k) const
{
    const Entry& e = get(k);
    if (e.kind != Entry::Block) fail(CFG_ESETUP, "dictionary: '" + k + "' is not a block");
    return *e.block;
}

double Dict::number(const std::string& k) const
{
    const Entry& e = get(k);
    if (e.kind != Entry::Number) fail(CFG_ESETUP, "dictionary: '" + k + "' is not a number");
    return e.number;
}

double Dict::numberOr(const std::string& k, double def) const { return has(k) ? number(k) : def; }

std::string Dict::word(const std::string& k) const
{
    const Entry& e = get(k);
    if (e.kind != Entry::Word && e.kind != Entry::Number) fail(CFG_ESETUP, "dictionary: '" + k + "' is not a word");
    return e.word;
}

std::string Dict::wordOr(const std::string& k, const std::string& def) const { return has(k) ? word(k) : def; }

std::vector<double> Dict::numbers(const std::string& k) const
{
    const Entry& e = get(k);
    if (e.kind != Entry::List) fail(CFG_ESETUP, "dictionary: '" + k + "' is not a list");
    std::vector<double> out;
    for (const auto& s : e.items)
    {
        double v;
        if (!isNumber(s, v)) fail(CFG_ESETUP, "dictionary: '" + k + "' holds a non-number");
        out.push_back(v);
    }
    return out;
}

}  // namespace cfg
