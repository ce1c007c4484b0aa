/* Stand-in for <re2/re2.h> so that the reference's statement.h / plan.h
 * compile without RE2. TEST INFRASTRUCTURE.
 *
 * The only patterns the reference builds are those of
 * Comparison::like_match (include/data_model/statement.h:119-158): a LIKE
 * pattern with '%' -> ".*", '_' -> "." and the regex metacharacters
 * escaped with a backslash. This stand-in matches exactly that subset with
 * RE2's default meaning (UTF-8 mode: "." is one code point other than a
 * newline), so the reference's scan filters can be run as a check of the
 * oracle's LIKE; any other pattern is refused (ok() == false, which
 * like_match turns into "no match"). */
#pragma once
#include <cstdint>
#include <string>
#include <string_view>
#include <vector>

class RE2 {
  public:
    struct Options {};
    RE2(const std::string &pattern, const Options &) {
        for (size_t i = 0; i < pattern.size(); ++i) {
            const char c = pattern[i];
            if (c == '\\') {
                if (i + 1 >= pattern.size()) { ok_ = false; return; }
                toks_.push_back({LIT, (uint8_t)pattern[++i]});
            } else if (c == '.') {
                if (i + 1 < pattern.size() && pattern[i + 1] == '*') {
                    toks_.push_back({STAR, 0});
                    ++i;
                } else {
                    toks_.push_back({ANY, 0});
                }
            } else if (c == '*' || c == '+' || c == '?' || c == '(' || c == ')' || c == '[' || c == ']' ||
                       c == '{' || c == '}' || c == '|' || c == '^' || c == '$') {
                ok_ = false; /* not a form like_match emits */
                return;
            } else {
                toks_.push_back({LIT, (uint8_t)c});
            }
        }
    }
    bool ok() const { return ok_; }
    const std::string &error() const { static const std::string e("unsupported pattern"); return e; }
    static bool FullMatch(std::string_view s, const RE2 &re) { return re.ok_ && re.match(s); }

  private:
    enum Kind { LIT, ANY, STAR };
    struct Tok { Kind k; uint8_t c; };
    std::vector<Tok> toks_;
    bool ok_ = true;
    static size_t cp(uint8_t b) {
        if (b < 0x80) return 1;
        if ((b & 0xE0) == 0xC0) return 2;
        if ((b & 0xF0) == 0xE0) return 3;
        if ((b & 0xF8) == 0xF0) return 4;
        return 1;
    }
    /* ok[i][j]: tokens j.. match text i.. */
    bool match(std::string_view s) const {
        const size_t n = s.size(), m = toks_.size();
        std::vector<uint8_t> ok((n + 1) * (m + 1), 0);
        auto at = [&](size_t i, size_t j) -> uint8_t & { return ok[i * (m + 1) + j]; };
        for (size_t i = n + 1; i-- > 0;)
            for (size_t j = m + 1; j-- > 0;) {
                if (j == m) { at(i, j) = i == n; continue; }
                const Tok &t = toks_[j];
                const uint8_t b = i < n ? (uint8_t)s[i] : 0;
                uint8_t r = 0;
                if (t.k == STAR) {
                    r = at(i, j + 1);
                    if (!r && i < n && b != '\n' && i + cp(b) <= n) r = at(i + cp(b), j);
                } else if (t.k == ANY) {
                    r = i < n && b != '\n' && i + cp(b) <= n && at(i + cp(b), j + 1);
                } else {
                    r = i < n && b == t.c && at(i + 1, j + 1);
                }
                at(i, j) = r;
            }
        return at(0, 0);
    }
};
