// Stand-in for boost::multiprecision::uint128_t, used only to compile the
// reference's own scalar operators as a test oracle.  The reference needs a
// fixed-width unsigned 128-bit integer that wraps modulo 2^128 (boost's
// `uint128_t` is `number<cpp_int_backend<128,128,unsigned,unchecked>>`), and
// `backend().size()` / `backend().limbs()` to read its 64-bit limbs.
#pragma once
#include <climits>
#include <cstdint>

namespace boost {
namespace multiprecision {

typedef unsigned long long limb_type;

class uint128_t {
    unsigned __int128 v_;
    mutable limb_type limbs_[2];  // refreshed by backend(); lives as long as *this

public:
    struct backend_view {
        const limb_type* l;
        unsigned size() const { return 2; }
        const limb_type* limbs() const { return l; }
    };

    uint128_t() : v_(0) {}
    uint128_t(unsigned __int128 v) : v_(v) {}
    uint128_t(unsigned long long v) : v_(v) {}
    uint128_t(unsigned long v) : v_(v) {}
    uint128_t(unsigned int v) : v_(v) {}
    uint128_t(unsigned short v) : v_(v) {}
    uint128_t(long long v) : v_((unsigned __int128)(__int128)v) {}
    uint128_t(long v) : v_((unsigned __int128)(__int128)v) {}
    uint128_t(int v) : v_((unsigned __int128)(__int128)v) {}

    backend_view backend() const {
        limbs_[0] = (limb_type)v_;
        limbs_[1] = (limb_type)(v_ >> 64);
        return backend_view{limbs_};
    }
    unsigned __int128 raw() const { return v_; }

    uint128_t& operator<<=(unsigned s) { v_ <<= s; return *this; }
    uint128_t& operator<<=(unsigned long s) { v_ <<= s; return *this; }
    uint128_t& operator+=(const uint128_t& o) { v_ += o.v_; return *this; }
    uint128_t& operator-=(const uint128_t& o) { v_ -= o.v_; return *this; }
    uint128_t& operator*=(const uint128_t& o) { v_ *= o.v_; return *this; }

    friend uint128_t operator+(const uint128_t& a, const uint128_t& b) { return uint128_t(a.v_ + b.v_); }
    friend uint128_t operator-(const uint128_t& a, const uint128_t& b) { return uint128_t(a.v_ - b.v_); }
    friend uint128_t operator*(const uint128_t& a, const uint128_t& b) { return uint128_t(a.v_ * b.v_); }
    friend uint128_t operator/(const uint128_t& a, const uint128_t& b) { return uint128_t(a.v_ / b.v_); }
    friend uint128_t operator%(const uint128_t& a, const uint128_t& b) { return uint128_t(a.v_ % b.v_); }
    friend bool operator<(const uint128_t& a, const uint128_t& b) { return a.v_ < b.v_; }
    friend bool operator>(const uint128_t& a, const uint128_t& b) { return a.v_ > b.v_; }
    friend bool operator<=(const uint128_t& a, const uint128_t& b) { return a.v_ <= b.v_; }
    friend bool operator>=(const uint128_t& a, const uint128_t& b) { return a.v_ >= b.v_; }
    friend bool operator==(const uint128_t& a, const uint128_t& b) { return a.v_ == b.v_; }
    friend bool operator!=(const uint128_t& a, const uint128_t& b) { return a.v_ != b.v_; }
};

}  // namespace multiprecision
}  // namespace boost
