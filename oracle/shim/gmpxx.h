// Test-infrastructure shim (oracle build only): GMP is not installed. psstest
// uses mpz_class only for its permutation hash, a product of 64-bit factors
// reduced modulo a 64-bit prime; every operand stays below 2^64, so a value
// type with 128-bit intermediate products covers that use.
#pragma once
#include <cstdint>
#include <cstdlib>
#include <ostream>

class mpz_class {
public:
    mpz_class() : v_(0) {}
    mpz_class(int x) : v_((uint64_t)(int64_t)x) {}
    mpz_class(unsigned long x) : v_(x) {}
    mpz_class(unsigned long long x) : v_(x) {}
    mpz_class(const char* s, int base) : v_(std::strtoull(s, nullptr, base)) {}
    mpz_class& operator=(int x) { v_ = (uint64_t)(int64_t)x; return *this; }
    mpz_class& operator*=(uint64_t x) { prod_ = (unsigned __int128)v_ * x; big_ = true; return *this; }
    mpz_class& operator%=(const mpz_class& p)
    {
        if (big_) { v_ = (uint64_t)(prod_ % p.v_); big_ = false; }
        else v_ %= p.v_;
        return *this;
    }
    bool operator==(const mpz_class& o) const { return value() == o.value(); }
    bool operator!=(const mpz_class& o) const { return !(*this == o); }
    bool operator==(int x) const { return value() == (unsigned __int128)(uint64_t)(int64_t)x; }
    bool operator!=(int x) const { return !(*this == x); }
    friend std::ostream& operator<<(std::ostream& os, const mpz_class& m) { return os << (unsigned long long)m.v_; }

private:
    unsigned __int128 value() const { return big_ ? prod_ : v_; }
    uint64_t v_;
    unsigned __int128 prod_ = 0;
    bool big_ = false;
};
