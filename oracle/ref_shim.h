/* Forced-include shim used only when compiling the upstream openntc sources
 * (libopenntc/*.cpp, ntc_kernel.cu) into oracle/_ref/ with g++/nvcc on Linux.
 *
 * The upstream sources were written against MSVC: they call std::sqrtf /
 * std::floorf (not declared in namespace std by libstdc++), use the MSVC
 * _countof macro, and rely on <cstdint> arriving transitively.  Nothing here
 * changes the upstream arithmetic; it only makes the translation units build.
 *
 * Test infrastructure: nothing in the product links against oracle/_ref.
 */
#pragma once
#ifdef __cplusplus
#include <cstdint>
#include <cmath>
#include <cstring>
namespace std {
using ::sqrtf;
using ::floorf;
}
#endif
#ifndef _countof
#define _countof(a) (sizeof(a) / sizeof((a)[0]))
#endif
