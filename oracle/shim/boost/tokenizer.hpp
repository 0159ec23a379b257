// Compatibility header for compiling the reference's CPU sources without Boost.
// Only what the reference's OBJ reader uses: boost::char_separator<char> (dropped and kept
// delimiters, empty fields dropped or kept) and boost::tokenizer over a std::string.
// The string is cut into fields at every delimiter; a kept delimiter is a token of its own;
// with keep_empty_tokens every field, empty or not, is a token.
#pragma once
#include <string>
#include <vector>
namespace boost {
enum empty_token_policy { drop_empty_tokens, keep_empty_tokens };
template <class Char>
class char_separator {
 public:
  explicit char_separator(const Char* dropped = " ", const Char* kept = "",
                          empty_token_policy empty = drop_empty_tokens)
      : dropped_(dropped ? dropped : ""), kept_(kept ? kept : ""), empty_(empty) {}
  std::vector<std::basic_string<Char>> split(const std::basic_string<Char>& s) const {
    std::vector<std::basic_string<Char>> out;
    std::basic_string<Char> field;
    auto flush = [&]() {
      if (!field.empty() || empty_ == keep_empty_tokens) out.push_back(field);
      field.clear();
    };
    for (Char ch : s) {
      if (dropped_.find(ch) != std::basic_string<Char>::npos) {
        flush();
      } else if (kept_.find(ch) != std::basic_string<Char>::npos) {
        flush();
        out.push_back(std::basic_string<Char>(1, ch));
      } else {
        field.push_back(ch);
      }
    }
    flush();
    return out;
  }
 private:
  std::basic_string<Char> dropped_, kept_;
  empty_token_policy empty_;
};
template <class Sep>
class tokenizer {
 public:
  typedef std::vector<std::string>::const_iterator iterator;
  tokenizer(const std::string& s, const Sep& sep) : tokens_(sep.split(s)) {}
  iterator begin() const { return tokens_.begin(); }
  iterator end() const { return tokens_.end(); }
 private:
  std::vector<std::string> tokens_;
};
}  // namespace boost
