/* Declarations of the six libzstd entry points that the ASZ reference calls.
 *
 * Test infrastructure only. The reference includes "../../third_party/zstd/lib/zstd.h"
 * (c_codes/asz_core/asz_param.hpp:249), but its zstd submodule is not checked out, so the
 * oracle build points that include at this file. The functions themselves come from the
 * system libzstd.so.1, which the recipe in oracle/Makefile links.
 */
#ifndef ASZ_ORACLE_ZSTD_DECLS_H
#define ASZ_ORACLE_ZSTD_DECLS_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
size_t ZSTD_compressBound(size_t srcSize);
size_t ZSTD_compress(void *dst, size_t dstCapacity, const void *src, size_t srcSize, int compressionLevel);
size_t ZSTD_decompress(void *dst, size_t dstCapacity, const void *src, size_t compressedSize);
unsigned long long ZSTD_getFrameContentSize(const void *src, size_t srcSize);
unsigned ZSTD_isError(size_t code);
const char *ZSTD_getErrorName(size_t code);
#ifdef __cplusplus
}
#endif
#endif
