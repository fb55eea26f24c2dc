// Sector keys of one or two 64-bit words.
//
// A configuration (c_0 .. c_{n-1}) is a mixed-radix number with the last site
// fastest.  When the product of the local dimensions is below 2^63 the key is
// one uint64 word (W = 1).  Otherwise (W = 2) the sites are split at n_hi:
// the high word holds the digits of sites [0, n_hi), the low word those of
// [n_hi, n), each a mixed-radix number below 2^63 with strides relative to its
// own word.  A two-word key is stored as 16 bytes, low word first, and is
// handled as the unsigned 128-bit integer hi * 2^64 + lo: since lo < 2^63 its
// numeric order is the lexicographic order of the configurations, the order
// of the reference's sorted uint16 tables.
//
// Per-digit work never divides a 128-bit number: a digit is taken from the
// one word that holds it, and a change of digit is added to that word only.
#pragma once
#include <cstdint>

namespace edg {

using u128 = unsigned __int128;

template <int W>
struct KeyOf;
template <>
struct KeyOf<1> {
  using type = uint64_t;
};
template <>
struct KeyOf<2> {
  using type = u128;
};

__device__ __forceinline__ uint64_t key_hi(uint64_t) { return 0; }
__device__ __forceinline__ uint64_t key_hi(u128 k) { return (uint64_t)(k >> 64); }
__device__ __forceinline__ uint64_t key_lo(uint64_t k) { return k; }
__device__ __forceinline__ uint64_t key_lo(u128 k) { return (uint64_t)k; }

// The word holding the digit of `site`.
__device__ __forceinline__ uint64_t key_word(uint64_t k, int, int) { return k; }
__device__ __forceinline__ uint64_t key_word(u128 k, int site, int n_hi) {
  return site < n_hi ? (uint64_t)(k >> 64) : (uint64_t)k;
}

// Key increment for a digit change worth `delta` (digit change times the
// site's stride, possibly negative) on `site`.  Added modulo 2^64 (2^128), it
// gives the exact key as long as the new digit is a valid state.
template <typename K>
__device__ __forceinline__ K key_step(int64_t delta, int site, int n_hi);
template <>
__device__ __forceinline__ uint64_t key_step<uint64_t>(int64_t delta, int, int) {
  return (uint64_t)delta;
}
template <>
__device__ __forceinline__ u128 key_step<u128>(int64_t delta, int site, int n_hi) {
  return site < n_hi ? ((u128)(uint64_t)delta) << 64 : (u128)(__int128)delta;
}

// Digit of `site` with stride `stride` (within its word) and dimension d.
template <typename K>
__device__ __forceinline__ int key_digit(K k, int site, int n_hi, uint64_t stride, uint64_t d) {
  return (int)((key_word(k, site, n_hi) / stride) % d);
}

// Loads and stores of key i of an array of W-word keys.
__device__ __forceinline__ uint64_t load_key(const uint64_t* __restrict__ keys, int64_t i, uint64_t*) {
  return __ldg(keys + i);
}
__device__ __forceinline__ u128 load_key(const uint64_t* __restrict__ keys, int64_t i, u128*) {
  const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(keys) + i);
  return ((u128)v.y << 64) | (u128)v.x;
}
template <typename K>
__device__ __forceinline__ K ld_key(const uint64_t* __restrict__ keys, int64_t i) {
  return load_key(keys, i, static_cast<K*>(nullptr));
}
__device__ __forceinline__ void st_key(uint64_t* keys, int64_t i, uint64_t k) { keys[i] = k; }
__device__ __forceinline__ void st_key(uint64_t* keys, int64_t i, u128 k) {
  reinterpret_cast<ulonglong2*>(keys)[i] = make_ulonglong2((uint64_t)k, (uint64_t)(k >> 64));
}

// Position of a key in the dense key space [0, prod d): the key itself for
// one word, hi * lo_space + lo for two (lo_space = product of the low word's
// dimensions).  Bucket tables index its top bits.
__device__ __forceinline__ u128 key_dense(uint64_t k, uint64_t) { return (u128)k; }
__device__ __forceinline__ u128 key_dense(u128 k, uint64_t lo_space) {
  return (u128)(uint64_t)(k >> 64) * lo_space + (uint64_t)k;
}

}  // namespace edg
