/* Stand-in for dm-heom/include/heom/integer_partition.hpp, whose common.hpp
 * pulls in Boost and noma submodules; declares the three functions of
 * dm-heom/src/heom/integer_partition.cpp (TEST INFRASTRUCTURE ONLY). */
#pragma once
#include <cstdint>
#include <memory>
namespace heom {
typedef std::int64_t int_t;
namespace ip {
int_t size_partiton_restrict(int_t n, int_t k);
int_t size_my_integer_partitions(int_t n, int_t s);
int_t my_integer_partitions(int_t n, int_t s, int_t* res);
}
}
