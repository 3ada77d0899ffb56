/*
 * Force-included (g++ -include) before the reference's Boost-free kernel
 * headers when oracle/ref_driver.cpp is compiled against the reference tree.
 * TEST INFRASTRUCTURE ONLY.
 *
 * It stands in for LibMIAUtil.h (which pulls in Boost, absent here) by
 * defining that header's include guard and the few names the kernels use:
 *   libmia_constexpr (LibMIAUtil.h: `#define libmia_constexpr constexpr`),
 *   restrict_libmia (a compiler restrict qualifier),
 *   boost::enable_if_c (IndexUtil.h:567, 591 use it for SFINAE only).
 * The reference headers themselves are compiled unmodified, in place.
 */
#ifndef LNT_REF_SHIM_H
#define LNT_REF_SHIM_H
#define LIBMIAUTIL_H 1
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <iostream>
#include <iterator>
#include <memory>
#include <type_traits>
#include <vector>
#define libmia_constexpr constexpr
#ifndef restrict_libmia
#define restrict_libmia __restrict__
#endif
namespace boost {
template <bool B, class T = void>
struct enable_if_c : std::enable_if<B, T> {};
}  // namespace boost
#endif
