// boost/dynamic_bitset.hpp — the part of boost::dynamic_bitset that the
// reference's src/FalconnPP.{h,cpp} use, written for this project so those
// files compile unchanged without Boost (TEST INFRASTRUCTURE ONLY: it builds
// the reference into oracle/_ref/ as a checker and CPU baseline).
//
// Semantics follow Boost's documentation: dynamic_bitset(n) holds n zero
// bits; operator[] gives a proxy that converts to bool, assigns from bool,
// and whose operator~ is the complement of the bit (a bool); find_first() /
// find_next(i) return the lowest set position (> i for find_next) or npos;
// clear() removes every bit (size 0).
#ifndef FPP_SHIM_BOOST_DYNAMIC_BITSET
#define FPP_SHIM_BOOST_DYNAMIC_BITSET

#include <climits>
#include <cstddef>
#include <memory>
#include <vector>

namespace boost {

template <typename Block = unsigned long, typename Allocator = std::allocator<Block>>
class dynamic_bitset {
 public:
  typedef std::size_t size_type;
  static const size_type npos = static_cast<size_type>(-1);
  static const int bits_per_block = (int)(sizeof(Block) * CHAR_BIT);

  class reference {
   public:
    reference(Block& b, Block m) : b_(&b), m_(m) {}
    operator bool() const { return (*b_ & m_) != 0; }
    bool operator~() const { return (*b_ & m_) == 0; }
    reference& operator=(bool x) {
      if (x)
        *b_ |= m_;
      else
        *b_ &= ~m_;
      return *this;
    }
    reference& operator=(const reference& r) { return *this = bool(r); }
    reference& flip() {
      *b_ ^= m_;
      return *this;
    }

   private:
    Block* b_;
    Block m_;
  };

  dynamic_bitset() : n_(0) {}
  explicit dynamic_bitset(size_type num_bits, unsigned long value = 0)
      : blocks_((num_bits + bits_per_block - 1) / bits_per_block, Block(0)), n_(num_bits) {
    for (size_type i = 0; i < num_bits && i < sizeof(unsigned long) * CHAR_BIT; ++i)
      if ((value >> i) & 1ul) (*this)[i] = true;
  }

  size_type size() const { return n_; }
  bool empty() const { return n_ == 0; }
  void clear() {
    blocks_.clear();
    n_ = 0;
  }

  reference operator[](size_type pos) { return reference(blocks_[pos / bits_per_block], mask(pos)); }
  bool operator[](size_type pos) const { return (blocks_[pos / bits_per_block] & mask(pos)) != 0; }
  bool test(size_type pos) const { return (*this)[pos]; }

  size_type find_first() const { return scan_from(0); }
  size_type find_next(size_type pos) const {
    if (pos == npos || pos + 1 >= n_) return npos;
    return scan_from(pos + 1);
  }

 private:
  static Block mask(size_type pos) { return Block(1) << (pos % bits_per_block); }

  size_type scan_from(size_type pos) const {
    if (pos >= n_) return npos;
    size_type b = pos / bits_per_block;
    Block w = blocks_[b] & (~Block(0) << (pos % bits_per_block));
    for (;;) {
      if (w) {
        const size_type r = b * bits_per_block + (size_type)__builtin_ctzll((unsigned long long)w);
        return r < n_ ? r : npos;
      }
      if (++b >= blocks_.size()) return npos;
      w = blocks_[b];
    }
  }

  std::vector<Block, Allocator> blocks_;
  size_type n_;
};

}  // namespace boost

#endif
