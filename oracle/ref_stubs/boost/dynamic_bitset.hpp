// Minimal stand-in for boost::dynamic_bitset, written for this repository so
// that the reference's ConvexPolyhedron2 (which stores its `outside` and `arcs`
// flags in a dynamic_bitset) compiles without Boost.  Only the members that
// ConvexPolyhedron2.tcc uses are provided: resize, set, test, operator[],
// none, count, find_first, operator~ and size.  Semantics follow Boost's
// documentation: resize() keeps the first bits and zero-fills new ones,
// find_first() returns npos when no bit is set, operator~ complements the
// bits inside size() only.
//
// Test infrastructure only: this header exists to build the compiled
// reference oracle under oracle/_ref.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace boost {

template <class Block = unsigned long>
class dynamic_bitset {
public:
    static constexpr std::size_t npos = static_cast<std::size_t>(-1);

    class reference {
    public:
        reference(std::vector<bool> &v, std::size_t i) : v_(v), i_(i) {}
        reference &operator=(bool b) { v_[i_] = b; return *this; }
        reference &operator=(const reference &r) { v_[i_] = bool(r); return *this; }
        operator bool() const { return v_[i_]; }
    private:
        std::vector<bool> &v_;
        std::size_t i_;
    };

    dynamic_bitset() = default;
    explicit dynamic_bitset(std::size_t n) : bits_(n, false) {}

    std::size_t size() const { return bits_.size(); }
    void resize(std::size_t n, bool value = false) { bits_.resize(n, value); }
    dynamic_bitset &set(std::size_t i, bool value = true) { bits_[i] = value; return *this; }
    bool test(std::size_t i) const { return bits_[i]; }
    bool operator[](std::size_t i) const { return bits_[i]; }
    reference operator[](std::size_t i) { return reference(bits_, i); }

    bool none() const {
        for (bool b : bits_) if (b) return false;
        return true;
    }
    std::size_t count() const {
        std::size_t c = 0;
        for (bool b : bits_) c += b;
        return c;
    }
    std::size_t find_first() const {
        for (std::size_t i = 0; i < bits_.size(); ++i) if (bits_[i]) return i;
        return npos;
    }
    dynamic_bitset operator~() const {
        dynamic_bitset r(*this);
        for (std::size_t i = 0; i < r.bits_.size(); ++i) r.bits_[i] = !r.bits_[i];
        return r;
    }

private:
    std::vector<bool> bits_;
};

}  // namespace boost
