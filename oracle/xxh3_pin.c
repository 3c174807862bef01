/* xxh3_pin.c — test infrastructure only: XXH3-64 with a caller's secret, from
   the xxHash header (0.8.x) that Apache Arrow vendors and pyarrow ships
   (arrow/vendored/xxhash/xxhash.h, the header qdb_string_hash_bytes includes,
   qdb/modules/qumirdb_runtime.cpp:6).  tests/test_string_hash.py builds it to
   pin the oracle's restatement of the string hash; nothing else uses it. */
#define XXH_INLINE_ALL
#include "arrow/vendored/xxhash/xxhash.h"

unsigned long long pin_xxh3_with_secret(const void* data, size_t size, const void* secret, size_t secret_size) {
    return XXH3_64bits_withSecret(data, size, secret, secret_size);
}
