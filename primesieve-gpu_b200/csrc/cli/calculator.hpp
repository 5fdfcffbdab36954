// calculator.hpp -- unsigned 64-bit integer expression evaluator for the CLI.
//
// Accepts what the reference CLI accepts for START / STOP / --dist values
// (include/primesieve/calculator.hpp, used by src/app/CmdOptions.cpp:193-196):
// decimal integers, "AeB" (A * 10^B), + - * / % ^ (power, right-assoc) and
// parentheses, e.g. "1e10", "2^64-1", "1e15+1e11". Any intermediate result
// outside [0, 2^64-1] is an error.
#pragma once
#include <cctype>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace psg {
namespace calculator {

class Parser {
public:
  explicit Parser(const std::string& s) : s_(s) {}

  uint64_t run() {
    skip();
    if (pos_ >= s_.size()) error("empty math expression");
    const uint64_t v = expr();
    skip();
    if (pos_ != s_.size()) error("unexpected character");
    return v;
  }

private:
  typedef unsigned __int128 u128;
  const std::string& s_;
  size_t pos_ = 0;

  [[noreturn]] void error(const std::string& what) const {
    throw std::runtime_error("Error: " + what + " at index " + std::to_string(pos_) +
                             " of math expression '" + s_ + "'");
  }
  [[noreturn]] void overflow(size_t at) {
    pos_ = at;
    error("64-bit unsigned integer overflow detected");
  }
  void skip() {
    while (pos_ < s_.size() && std::isspace((unsigned char) s_[pos_])) pos_++;
  }
  bool eat(char c) {
    skip();
    if (pos_ < s_.size() && s_[pos_] == c) { pos_++; return true; }
    return false;
  }
  uint64_t check(u128 v, size_t at) {
    if (v > (u128) ~(uint64_t) 0) overflow(at);
    return (uint64_t) v;
  }
  uint64_t pow(uint64_t b, uint64_t e, size_t at) {
    u128 r = 1;
    for (uint64_t i = 0; i < e; i++) {
      r *= b;
      if (r > (u128) ~(uint64_t) 0) overflow(at);
      if (b <= 1) break;
    }
    return (uint64_t) r;
  }
  uint64_t expr() {
    uint64_t v = term();
    for (;;) {
      const size_t at = pos_;
      if (eat('+')) v = check((u128) v + term(), at);
      else if (eat('-')) {
        const uint64_t r = term();
        if (r > v) { pos_ = at; error("negative result"); }
        v -= r;
      } else return v;
    }
  }
  uint64_t term() {
    uint64_t v = power();
    for (;;) {
      const size_t at = pos_;
      if (eat('*')) v = check((u128) v * power(), at);
      else if (eat('/')) {
        const uint64_t r = power();
        if (!r) { pos_ = at; error("division by zero"); }
        v /= r;
      } else if (eat('%')) {
        const uint64_t r = power();
        if (!r) { pos_ = at; error("division by zero"); }
        v %= r;
      } else return v;
    }
  }
  uint64_t power() {
    const uint64_t b = unary();
    const size_t at = pos_;
    if (eat('^')) return pow(b, power(), at);
    return b;
  }
  uint64_t unary() {
    if (eat('+')) return unary();
    if (eat('-')) {
      const uint64_t v = unary();
      if (v) error("negative result");
      return 0;
    }
    return primary();
  }
  uint64_t primary() {
    skip();
    if (eat('(')) {
      const uint64_t v = expr();
      if (!eat(')')) error("missing ')'");
      return v;
    }
    if (pos_ >= s_.size() || !std::isdigit((unsigned char) s_[pos_])) error("expected a number");
    const size_t at = pos_;
    u128 v = 0;
    while (pos_ < s_.size() && std::isdigit((unsigned char) s_[pos_])) {
      v = v * 10 + (uint64_t) (s_[pos_++] - '0');
      if (v > (u128) ~(uint64_t) 0) overflow(at);
    }
    // scientific notation: AeB = A * 10^B
    if (pos_ < s_.size() && (s_[pos_] == 'e' || s_[pos_] == 'E')) {
      pos_++;
      if (pos_ >= s_.size() || !std::isdigit((unsigned char) s_[pos_])) error("expected an exponent");
      uint64_t e = 0;
      while (pos_ < s_.size() && std::isdigit((unsigned char) s_[pos_])) {
        e = e * 10 + (uint64_t) (s_[pos_++] - '0');
        if (e > 1000) overflow(at);
      }
      v = (u128) check(v, at) * pow(10, e, at);
    }
    return check(v, at);
  }
};

inline uint64_t eval_u64(const std::string& s) { return Parser(s).run(); }

} // namespace calculator
} // namespace psg
