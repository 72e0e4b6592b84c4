// Minimal stand-in for boost::dynamic_bitset<>, used only to compile the
// reference search sources into the reference binaries under oracle/_ref.
// Boost is not installed in this image. The reference uses: a sized
// constructor with an optional initial value (brace-initialised as
// `flags{n, 0}`), operator[] for read and write, reset(), resize(), size().
// There is deliberately no initializer_list constructor, so `{n, 0}` picks
// the sized constructor.
#ifndef PANNS_ORACLE_SHIM_DYNAMIC_BITSET_HPP
#define PANNS_ORACLE_SHIM_DYNAMIC_BITSET_HPP

#include <cstddef>
#include <cstdint>
#include <vector>

namespace boost {

template <typename Block = unsigned long>
class dynamic_bitset {
public:
    class reference {
    public:
        reference(std::uint64_t *w, std::uint64_t m) : w_(w), m_(m) {}
        operator bool() const { return (*w_ & m_) != 0; }
        reference &operator=(bool v) {
            if (v) *w_ |= m_; else *w_ &= ~m_;
            return *this;
        }
        reference &operator=(int v) { return *this = (v != 0); }
        reference &operator=(const reference &o) { return *this = bool(o); }
    private:
        std::uint64_t *w_;
        std::uint64_t m_;
    };

    dynamic_bitset() = default;
    explicit dynamic_bitset(std::size_t n, unsigned long value = 0)
        : n_(n), words_((n + 63) / 64, 0) {
        if (value && n_) words_[0] = value;
    }

    std::size_t size() const { return n_; }
    void resize(std::size_t n) { n_ = n; words_.resize((n + 63) / 64, 0); }
    dynamic_bitset &reset() {
        for (auto &w : words_) w = 0;
        return *this;
    }
    bool operator[](std::size_t i) const { return (words_[i >> 6] >> (i & 63)) & 1u; }
    reference operator[](std::size_t i) {
        return reference(&words_[i >> 6], std::uint64_t(1) << (i & 63));
    }

private:
    std::size_t n_ = 0;
    std::vector<std::uint64_t> words_;
};

} // namespace boost

#endif
