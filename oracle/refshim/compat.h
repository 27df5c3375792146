// Force-included (-include) when compiling the reference Core with GCC 13.
// Test infrastructure only.
//  * <cstdint>: Core/DER/Definitions.h uses uint32_t without including it.
//  * std::swap on two std::vector<bool>::reference proxies (Core/TwoDScene.cpp
//    swapParticles swaps m_twist / m_is_strand_tip elements): libstdc++ 13 only
//    provides swap(_Bit_reference, _Bit_reference) overloads that GCC 13 no
//    longer picks for the rvalue proxies, so add one that exchanges the bits.
#ifndef WCREF_COMPAT_H
#define WCREF_COMPAT_H
#ifdef __cplusplus
#include <cstdint>
#include <vector>
namespace std {
template <class B = _Bit_reference>
inline void swap(B a, _Bit_reference b) noexcept {
  bool t = a;
  a = bool(b);
  b = t;
}
}  // namespace std
#endif
#endif
