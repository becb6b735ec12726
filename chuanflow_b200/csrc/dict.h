// Case-dictionary reader for the reference's case.dict grammar
// (src/common/include/cf/common/Dictionary.h:13-30): `key value;`,
// `key (a b c);`, `key { ... }`, quoted strings, '#' and '//' comments.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace cfg
{

class Dict
{
public:
    struct Entry
    {
        enum Kind { Number, Word, List, Block } kind = Word;
        double number = 0;
        std::string word;
        std::vector<std::string> items;  // list items as written
        std::shared_ptr<Dict> block;
    };

    static Dict parse(const std::string& text);
    static Dict parseFile(const std::string& path);

    bool has(const std::string& k) const { return entries_.count(k) > 0; }
    const std::vector<std::string>& keys() const { return order_; }
    const Dict& dict(const std::string& k) const;
    double number(const std::string& k) const;
    double numberOr(const std::string& k, double def) const;
    std::string word(const std::string& k) const;
    std::string wordOr(const std::string& k, const std::string& def) const;
    std::vector<double> numbers(const std::string& k) const;

private:
    const Entry& get(const std::string& k) const;
    std::map<std::string, Entry> entries_;
    std::vector<std::string> order_;
    friend struct DictParser;
};

}  // namespace cfg
