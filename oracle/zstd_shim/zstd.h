/*
 * Oracle test infrastructure only.
 *
 * Prototype-only stand-in for the zstd header, so that the reference's disk
 * tier (util.c, which includes <zstd.h>) compiles in an image that ships the
 * zstd runtime but not its development header.  Only the five entry points
 * the reference's util.c calls are declared (util.c:218-255).  The oracle
 * harness never touches the disk tier, so it links stub definitions from
 * ref_harness.c; the full reference binary built for the KRvK known-answer
 * run links the real libzstd.so.1 by path instead.
 */
#ifndef ORACLE_ZSTD_SHIM_H
#define ORACLE_ZSTD_SHIM_H

#include <stddef.h>

typedef struct ZSTD_CCtx_s ZSTD_CCtx;
typedef struct ZSTD_DCtx_s ZSTD_DCtx;

size_t ZSTD_compressBound(size_t srcSize);
ZSTD_CCtx *ZSTD_createCCtx(void);
ZSTD_DCtx *ZSTD_createDCtx(void);
size_t ZSTD_compressCCtx(ZSTD_CCtx *cctx, void *dst, size_t dstCapacity,
                         const void *src, size_t srcSize, int compressionLevel);
size_t ZSTD_decompressDCtx(ZSTD_DCtx *dctx, void *dst, size_t dstCapacity,
                           const void *src, size_t srcSize);

#endif
