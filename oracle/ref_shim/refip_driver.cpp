/* C entry point to the reference's integer_partition.cpp compiled as is
 * (TEST INFRASTRUCTURE ONLY). */
#include <cstdint>
#include "heom/integer_partition.hpp"

extern "C" int64_t refip_integer_partitions(int32_t n, int32_t s, int64_t* out, int64_t cap)
{
    int64_t count = heom::ip::size_my_integer_partitions(n, s);
    if (count > cap) return -1;
    return heom::ip::my_integer_partitions(n, s, out);
}
