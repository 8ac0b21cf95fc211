// Stand-in for the boost::tokenizer / char_separator pair the engine splits
// argument strings and scene-file lines with: separator characters are
// dropped and empty tokens skipped (char_separator's default behaviour).
#pragma once
#include <string>
#include <vector>

namespace boost {

template <class Char = char>
class char_separator {
public:
    explicit char_separator(const Char *dropped = 0) : dropped_(dropped ? dropped : "") {}
    bool is_sep(Char c) const { return dropped_.find(c) != std::basic_string<Char>::npos; }

private:
    std::basic_string<Char> dropped_;
};

template <class Sep = char_separator<char>, class It = std::string::const_iterator, class Tok = std::string>
class tokenizer {
public:
    typedef typename std::vector<Tok>::const_iterator iterator;
    typedef iterator const_iterator;
    tokenizer(const std::string &text, const Sep &sep)
    {
        Tok cur;
        for (char c : text) {
            if (sep.is_sep(c)) {
                if (!cur.empty()) tokens_.push_back(cur);
                cur.clear();
            } else {
                cur.push_back(c);
            }
        }
        if (!cur.empty()) tokens_.push_back(cur);
    }
    iterator begin() const { return tokens_.begin(); }
    iterator end() const { return tokens_.end(); }

private:
    std::vector<Tok> tokens_;
};

}  // namespace boost
