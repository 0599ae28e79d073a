/* Stand-in for lz4's header (the library is on the system, its header is not), for
 * building the reference's super k-mer chunk compression here: the three entry points
 * it calls, as lz4's public API declares them (lz4.h, BSD-2-Clause).  Test and
 * baseline infrastructure only. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
int LZ4_compressBound(int inputSize);
int LZ4_compress_default(const char* src, char* dst, int srcSize, int dstCapacity);
int LZ4_decompress_safe(const char* src, char* dst, int compressedSize, int dstCapacity);
#ifdef __cplusplus
}
#endif
