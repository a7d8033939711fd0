/*
 * tbgpu -- B200 (sm_100a) engine for the per-king-slice ply step of the
 * tb8gen retrograde generator, behind a plain C ABI.
 *
 * The reference runs its ply step as `static` workers driven by
 * run_threaded(worker, work, false) (threads.c:266-289), with parameters in
 * file-scope globals (g_pos, ii, capt_ii, pc_to_set, work_slice, ...) and
 * the slice buffers in kslice_buf[]/kslice_sub_buf[] addressed through
 * kslice_slot[] (kslice.c:23-28).  Each entry point below replaces one such
 * call; the host schedule (calc_W_n / calc_L_n, tb8gen.c:943-1084) stays.
 *
 * Conventions
 *  - Every function returns TBG_OK (0) or a negative tbg_status.  The
 *    reference exits on failure; its host shim does exit(EXIT_FAILURE) on a
 *    negative status.
 *  - Bitmaps use the reference's byte layout: one bit per position,
 *    LSB-first within bytes (kslice.h:30-55), rounded up to 64 bytes
 *    (kslice.c:191-196).  Device pointers must be 16-byte aligned.
 *  - The caller owns all device memory (it binds it with tbg_slot_bind /
 *    tbg_sub_bind); the library allocates only its own small status and
 *    counter words (and, in tbg_ply_batch, a work queue).
 *  - Work is stream-ordered on the stream set by tbg_set_stream (default:
 *    the legacy default stream).  Calls that return a count synchronise
 *    with a bounded wait.  One host thread per library instance, like the
 *    reference's single calling thread.
 *  - Positions are indexed with 32-bit arithmetic when the slice size is
 *    below 2^32 and 64-bit arithmetic otherwise.
 */
#ifndef TBGPU_H
#define TBGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum tbg_status {
  TBG_OK = 0,
  TBG_ERR_ARG = -1,      /* invalid argument or misaligned pointer */
  TBG_ERR_STATE = -2,    /* tbg_init not called / no material selected */
  TBG_ERR_UNBOUND = -3,  /* a slice the call reads or writes has no bound buffer */
  TBG_ERR_CUDA = -4,     /* CUDA runtime error (see tbg_last_error) */
  TBG_ERR_NOMEM = -5,    /* the library could not allocate its own device words */
  TBG_ERR_DEVICE = -6,   /* a kernel met an access outside the bound buffers and skipped it */
  TBG_ERR_TIMEOUT = -7,  /* a bounded wait gave up; the stream may still be running */
  TBG_ERR_RANGE = -8     /* a size beyond a stated limit */
};

/* struct IdxInfo, tb8gen.h:4-13 (same field order and types). */
typedef struct tbg_idx_info {
  int numsets;
  uint64_t size;
  uint64_t factor[6];
  uint32_t subfactor[6];
  int first[6];
  int mult[6];
  int last[6];
} tbg_idx_info;

/* struct Position, movegen.h:18-26, pawnless build (same layout). */
typedef struct tbg_position {
  uint64_t occ;
  uint8_t sq[8], pt[8];
  int num, stm;
  int8_t pcs[2][8];
} tbg_position;

/* ---- set-up ---------------------------------------------------------- */

/* Replaces the table set-up of main() (init_movegen, init_tables,
 * init_indices; tb8gen.c:1279-1282): selects device 0 (or the current
 * device) and uploads nothing yet.  Idempotent. */
int tbg_init(void);

/* Registers a material from the reference's own set-up (ii, capt_ii[],
 * g_pos, pc_to_set: tb8gen.c:1329-1378).  ii->subfactor[0] may carry the
 * reference's +64 guard (tb8gen.c:227).  Returns a material handle >= 0
 * and makes it current, or a negative status. */
int tbg_material_init(const tbg_idx_info *ii, const tbg_idx_info *capt_ii,
                      const tbg_position *pos, const int *pc_to_set);

/* Same, parsing a material string such as "KRRRvKRRR" exactly as main()
 * does (tb8gen.c:1284-1378).  Returns a handle >= 0 or a negative status. */
int tbg_material_from_name(const char *name);

/* Makes material `mat` current for the per-slice calls. */
int tbg_material_select(int mat);

/* Geometry of the current material: slice size in positions, slice bitmap
 * bytes (kslice_cache_lines << 6), sub buffer bytes per slice
 * (max of sub_size[], kslice.c:219) and the byte offset of set k in it
 * (sub_offset[], kslice.c:214-218). */
int tbg_geometry(uint64_t *size, uint64_t *bytes, uint64_t *sub_bytes,
                 uint64_t sub_offset[6], uint64_t capt_size[6]);

/* Stream for all following work (a cudaStream_t; NULL = default). */
int tbg_set_stream(void *stream);

/* Seed and modulus (3 or 5) of the 7-piece WDL stub used by tbg_calc_sub. */
int tbg_set_stub(uint64_t seed, int modulus);

/* Device memory for a C host that binds its own slices (kslice_setup's
 * alloc_huge, kslice.c:198-227): zero-filled, 256-byte aligned.
 * TBG_ERR_NOMEM when the device cannot hold it, where the reference exits
 * (out_of_mem, util.c:111-115).  For tests of that path, the environment
 * variable TBG_FAIL_ALLOC_AT=k (read by tbg_init) makes the k-th call of
 * tbg_alloc / tbg_host_alloc in the process fail that way. */
int tbg_alloc(size_t bytes, void **dev);
int tbg_free(void *dev);

/* Copies between host memory and device memory on the library's stream,
 * returning when the copy is done: the host tier of a C host that keeps
 * slices in host memory (in place of kslice_read / kslice_write,
 * kslice.c:317-379). */
int tbg_copy_to_device(void *dev, const void *host, size_t bytes);
int tbg_copy_to_host(void *host, const void *dev, size_t bytes);

/* The same copies queued on the library's stream without waiting (ordered
 * with the kernels there; the host memory must stay untouched until a
 * tbg_sync).  From page-locked memory (tbg_host_alloc) they run at full
 * link speed. */
int tbg_copy_to_device_async(void *dev, const void *host, size_t bytes);
int tbg_copy_to_host_async(void *host, const void *dev, size_t bytes);

/* Page-locked host memory for a host tier (TBG_ERR_NOMEM when the host
 * cannot lock that much; fall back to ordinary memory then). */
int tbg_host_alloc(size_t bytes, void **host);
int tbg_host_free(void *host);

/* ---- host-tier copies on their own streams (no counterpart in the
 * reference, whose worker threads read and write the slice files between
 * run_threaded calls, kslice.c:317-379) ----------------------------------
 * Inbound and outbound copies run on two streams of the library, apart from
 * the library stream that runs the kernels, so a host tier can fetch the
 * next slices and write back the last ones while the kernels run.  They are
 * ordered by tickets: a ticket stands for a point of one stream and is live
 * until 8192 newer tickets exist (TBG_ERR_ARG for a dead one). */

/* Ticket of the library stream's current point (the work issued so far). */
int tbg_mark(uint64_t *ticket);

/* Host-to-device / device-to-host copy on the inbound / outbound stream,
 * started after the point of ticket `after` (0: no wait; the stream keeps
 * its order, so later copies wait as well).  bytes may be 0: a pure wait.
 * With ticket != NULL, reports the ticket of the point after the copy. */
int tbg_copy_in(void *dev, const void *host, size_t bytes, uint64_t after, uint64_t *ticket);
int tbg_copy_out(void *host, const void *dev, size_t bytes, uint64_t after, uint64_t *ticket);

/* Later work on the library stream waits for the ticket's point. */
int tbg_join(uint64_t ticket);

/* The host waits (bounded: timeout_ms, 0 = 600000) for the ticket's point. */
int tbg_wait_ticket(uint64_t ticket, int timeout_ms);

/* ---- slot map (kslice_slot / kslice_buf / kslice_sub_buf) ------------ */

/* Binds a device bitmap of `bytes` bytes to slice s of the current
 * material; s == -1 is the scratch slot (kslice_buf[19]).  NULL unbinds. */
int tbg_slot_bind(int s, void *dev_bitmap, size_t bytes);

/* Binds a device sub buffer (the five sub bitmaps of kslice_sub_buf use
 * this layout: sets at sub_offset[k]) to slice s; s == -1 is the scratch
 * slot's sub base (kslice_sub_get_base(-1), kslice.h:63-68). */
int tbg_sub_bind(int s, void *dev_sub, size_t bytes);

int tbg_unbind_all(void);

/* ---- the ply step ---------------------------------------------------- */

/* predecessors(stm, s), tb8gen.c:519-527: every set bit of the scratch
 * slot (opponent to move, slice s) is unmoved by side stm; marks are ORed
 * into slice s and the slices its king moves reach (all must be bound). */
int tbg_predecessors(int stm, int s);

/* The candidates phase of calc_L_n (tb8gen.c:951-997) for a host that
 * verifies them next against the same "wins": predecessors(stm, s) where
 * a predecessor that a quiet move of the unmoved slider (one square along
 * its ray) takes to a position outside the opponent's "wins" of slice s
 * (opp_wins, bytes >= the slice bitmap) is not marked in slice s -- it
 * cannot survive check_successors (check_moves, tb8gen.c:594-602).  The
 * verified losses are the reference's; the candidates are a subset of
 * predecessors()'s.  No counterpart in the reference: it marks every
 * predecessor and verifies all of them. */
int tbg_candidates(int stm, int s, const void *opp_wins, size_t bytes);

/* predecessors_sub(stm, s, legality), tb8gen.c:397-414: uncaptures from
 * the sub buffer bound to s (sets of colour stm^1) into slice s and its
 * king-move slices. */
int tbg_predecessors_sub(int stm, int s, int legality);

/* check_successors(stm, s), tb8gen.c:653-661: candidates in the scratch
 * slot are kept iff legal and every move leads to a bit set in the
 * opponent's "wins" bound to s (and its king-move slices) or, for a
 * capture, in the sub buffer bound there. */
int tbg_check_successors(int stm, int s);

/* check_successors with the survivors written to dev_out (the bound
 * bitmap size) instead of in place; the candidates are left unchanged.
 * In the reference the in-place result is written out as L (tb8gen.c:1014-1017). */
int tbg_check_successors_to(int stm, int s, void *dev_out);

/* calc_sub_kslices for one slice (tb8gen.c:327-335): the five capture
 * classes loss, bloss, draw, cwin, win of every set of colour stm, each
 * into its own device buffer of sub_bytes, sets at sub_offset[k].  The
 * 7-piece values come from the seeded stub (tbg_set_stub). */
int tbg_calc_sub(int stm, int s, void *const dev_cls[5]);

/* Illegal-position masks of slice s (calc_illegal_worker,
 * tb8gen.c:734-745): for white and for black to move. */
int tbg_calc_illegal(int s, void *dev_ill_w, void *dev_ill_b);

/* Mates (L0) of slice s (calc_mate_worker, tb8gen.c:752-758). */
int tbg_calc_mate(int s, const void *dev_ill_w, const void *dev_ill_b,
                  void *dev_mate_w, void *dev_mate_b);

/* W-step epilogue (tb8gen.c:1072-1077), fused: T(s) &= ~wins(s_wins);
 * *cnt = popcount below the slice size; wins(s_wins) |= T(s).  s_wins is
 * usually -1.  With cnt != NULL the call waits (bounded) for the count. */
int tbg_epilogue_W(int s, int s_wins, uint64_t *cnt);

/* Out-of-place epilogue: T(s) &= ~wins_in; wins_out = wins_in | T(s).
 * wins_in == wins_out is tbg_epilogue_W.  The reference reads "wins" from
 * disk into the scratch slot and writes it back (tb8gen.c:1072-1077); with
 * HBM-resident bitmaps the old and new "wins" can be separate buffers. */
int tbg_epilogue_W_to(int s, const void *dev_wins_in, void *dev_wins_out,
                      uint64_t *cnt);

/* kslice_count(s), kslice.c:524-527 (waits, bounded). */
int tbg_count(int s, uint64_t *cnt);

/* kslice_count (kslice.c:524-527) summed over n bitmaps of the bound size
 * at dev_base + i * stride_bytes (the slices of one plane), in one launch;
 * no counterpart in the reference, which counts slice by slice.  dev_base
 * 16-byte aligned, stride_bytes a multiple of 16 and at least the bitmap
 * size, 1 <= n <= 65535.  Waits (bounded) for the count. */
int tbg_count_strided(const void *dev_base, uint64_t stride_bytes, int n, uint64_t *cnt);

/* kslice_clear(s), kslice.c:292-296. */
int tbg_clear(int s);

/* kslice_sub_and_not(s1, s2, stm), kslice.c:481-487. */
int tbg_sub_and_not(int s1, int s2, int stm);

/* ---- batched ply (persistent kernel) ---------------------------------- */

/* Starts recording: the following ply-step calls (tbg_predecessors,
 * tbg_predecessors_sub, tbg_check_successors[_to], tbg_epilogue_W[_to] with
 * cnt == NULL, tbg_clear) are checked and recorded with their current
 * bindings instead of launched.  No counterpart in the reference, whose
 * schedule runs one run_threaded call at a time (threads.c:266-289). */
int tbg_batch_begin(void);

/* Ends recording and uploads the batch (the library allocates its work
 * queue here).  Reports the number of recorded calls and of work items. */
int tbg_batch_end(int *nops, uint64_t *nitems);

/* Runs the recorded batch on the current stream: mode 0 launches one kernel
 * per recorded call in record order (the plain path); mode 1 runs all of
 * them in one persistent kernel fed by a device work queue, each call
 * starting tile by tile as soon as the calls it depends on (by buffer) are
 * done; mode 2 is the same persistent kernel with every work item cut into
 * one part per warp, each warp taking parts on its own (no block barrier
 * between a tile's sources).  All give the same bitmaps as the calls made
 * one by one. */
int tbg_batch_run(int mode);

/* Epilogue counts of the last run, in record order (waits, bounded). */
int tbg_batch_counts(uint64_t *out, int n);

/* Records, in a batch, the count of the bitmap bound to s (kslice_count,
 * kslice.c:524-527) after the recorded calls that write it.  Its value comes
 * from tbg_batch_counts[_async] in record order, among the epilogue counts.
 * TBG_ERR_STATE outside a recording. */
int tbg_batch_count(int s);

/* Queues the copy of the first n counts of the last run into host memory
 * on the library stream (asynchronous when host_out is page-locked); the
 * values are there once the stream has passed this point (tbg_sync, or a
 * ticket marked after it). */
int tbg_batch_counts_async(uint64_t *host_out, int n);

/* Selects one of 4 batch slots (default 0); tbg_batch_begin .. counts act
 * on the selected slot, and every slot keeps its recorded batch and work
 * queue, so a caller can alternate steps recorded over different buffers
 * (one step's copies overlapping the other's kernels).  TBG_ERR_STATE while
 * a batch is being recorded. */
int tbg_batch_select(int slot);

/* Work-item shape of the scatters, in tiles of 32,768 positions per item of
 * the persistent queue and per block of a plain launch: scatter_tiles for
 * tbg_predecessors (0: 1), candidate_tiles for tbg_candidates (0: 4).  A
 * block gathers the sources of an item's tiles before handing them out to
 * its threads.  Applies to later recordings and re-cuts the selected
 * recorded batch (*nitems: its work items now, 0 if none is recorded;
 * nitems may be NULL).  Results do not depend on it.  No counterpart in the
 * reference (its g_total_work ranges, tb8gen.c:1327, are the nearest
 * knob). */
int tbg_batch_shape(int scatter_tiles, int candidate_tiles, uint64_t *nitems);

/* Persistent-launch configuration of every slot: CTAs per SM (default 4),
 * and the iteration bound of a dependency wait (<= 0 keeps the current
 * one). */
int tbg_batch_tune(int ctas_per_sm, long long spin_limit);

/* dst = a & ~b over `bytes` (a multiple of 16) of explicit device buffers:
 * kslice_and_not / kslice_sub_and_not (kslice.c:352-368, 481-487) for a
 * host that keeps its bitmaps outside the slot map. */
int tbg_bitmap_and_not(void *dst, const void *a, const void *b, size_t bytes);

/* Waits (bounded: timeout_ms, 0 = 600000) for the stream; reports a kernel
 * status word (TBG_ERR_DEVICE) if one was raised since the last wait. */
int tbg_sync(int timeout_ms);

/* Last error text (CUDA or argument detail). */
const char *tbg_last_error(void);

/* Number of kernels this library has launched so far (instrumentation). */
int tbg_launches(uint64_t *n);

/* ---- epilogue without allocation (no counterpart in the reference) ---- */

/* The fused W-step epilogue of tbg_epilogue_W_to on raw device pointers, for
 * callers that cannot allocate device memory: processes whose HBM is all
 * owned by a caching allocator or a fixed-budget pool, and foreign-language
 * hosts whose bindings forbid a library to allocate.  It needs no tbg_init
 * (which allocates) and calls no allocating routine; its scratch is a static
 * 8 KiB device array held by every GPU that loads the library.
 *   T &= ~wins_in;  wins_out = wins_in | T;  *cnt = popcount of T below nbits
 * wins_in may equal wins_out.  `bytes` (a multiple of 16) is the bitmap size;
 * at most 1 GiB (TBG_ERR_RANGE beyond).  The first call on a device looks up
 * the scratch address on that device; make it before any stream capture.
 * The address is kept for the life of the device's primary context (not
 * valid after a cudaDeviceReset).  Calls share the scratch: calls that
 * overlap on the GPU race and must not be issued.  Waits for the stream
 * before returning the count. */
int tbg_epilogue_W_static(void *dev_T, const void *dev_wins_in, void *dev_wins_out,
                          uint64_t nbits, uint64_t bytes, void *stream,
                          uint64_t *cnt);

/* ---- 7-piece WDL table probes --------------------------------------- */

/* A probe query: the squares of the position's pieces, in the material's
 * piece order (the order of main(), tb8gen.c:1331-1339: white king, black
 * king, then knights, bishops, rooks, queens, each type white before
 * black), and the side to move (0 white, 1 black).  16 bytes, like the
 * reference Position's sq[]/stm fields (movegen.h) that probe_table reads.
 * Query arrays passed to the probe and encode calls start on a 16-byte
 * boundary (TBG_ERR_ARG otherwise): each query is read as one vector. */
typedef struct {
  uint8_t sq[8];
  uint8_t stm;
  uint8_t pad[7];
} tbg_query;

/* Builds the synthetic WDL table of a pawnless material in the reference's
 * .rtbw layout, as init_table (probe.c:1210-1344) parses it: magic,
 * split flag, per-side piece header, setup_pairs bytes (rANS, 64 KiB
 * blocks, idx_bits 16), frequency table (write_freq_table, rans.c:239-276),
 * sympat, index table, size table, 64-byte aligned rANS blocks.  Position
 * idx of side bside holds wdl = VALS[splitmix64(seed ^ idx ^ bside << 63)
 * mod modulus], VALS = {-2, 0, 2} (modulus 3) or {-2..2} (modulus 5).
 * The reference has no table writer; this is the writer its reader reads.
 * on_device != 0: *table is device memory (cudaMalloc; release it with
 * tbg_free), built by kernels; else host memory (tbg_table_free_host),
 * built on the CPU for small materials.  *bytes is the file size. */
int tbg_table_build(const char *material, uint64_t seed, int modulus, int on_device,
                    void **table, uint64_t *bytes);
int tbg_table_free_host(void *table);

/* Opens a table image resident in device memory (the reference maps the
 * file, map_tb / init_table, probe.c:107, 1210).  At most 8 open tables.
 * Only rANS-compressed pawnless WDL tables are read (the format of
 * tbg_table_build); other layouts return TBG_ERR_ARG. */
int tbg_probe_open(const void *dev_table, uint64_t bytes, const char *material, int *handle);
int tbg_probe_close(int handle);

/* probe_table(pos, 0, WDL) (probe.c:1522-1597) for n device-resident
 * queries: dev_out[i] = the table's wdl (-2..2) of query i.
 * mode 0: queries grouped by rANS block, each touched block decoded once
 * (falls back to mode 1 for tables whose symbols cover unequal position
 * counts); mode 1: each query decoded on its own, as decompress_rans
 * (probe.c:1346-1390) does.  Both give identical results.  Work is queued
 * on the library's stream; the call returns without waiting when the
 * scratch budget (tbg_probe_tune) holds min(n, table blocks) blocks, else it
 * waits once to plan decode waves.  A handle's scratch serves every batch
 * on it: batches on one handle must not overlap on the GPU (keep them on one
 * stream, or open one handle per concurrent stream). */
int tbg_probe_wdl_batch(int handle, const void *dev_queries, uint64_t n, void *dev_out, int mode);

/* tbg_probe_wdl_batch on compact queries of 8 bytes (materials of at most 7
 * pieces): the squares in bytes 0-6 in the order of tbg_query, the side to
 * move in byte 7; the array 8-byte aligned.  Half the bytes a host feeds per
 * position; same results.  No counterpart in the reference. */
int tbg_probe_wdl_batch8(int handle, const void *dev_queries, uint64_t n, void *dev_out, int mode);

/* Where side `side` of an open table keeps its rANS blocks: byte offset of
 * block 0 in the image (block k at data_offset + k * 65536), the number of
 * blocks and of positions (init_table's walk, probe.c:1304-1331). */
int tbg_probe_layout(int handle, int side, uint64_t *data_offset, uint64_t *nblocks,
                     uint64_t *positions);

/* Bytes of one side's compressed streams: per block, from the stream's
 * first word (its first nonzero 32-bit word, where decompress_rans starts,
 * probe.c:1362-1372) to the block's end, summed.  tbg_probe_open finds
 * every block's start once, so that decodes skip the zero padding in front
 * of the streams; no counterpart in the reference. */
int tbg_probe_stream_bytes(int handle, int side, uint64_t *bytes);

/* Device time of the phases of the handle's last grouped batch (CUDA
 * events on the library's stream): ms[0] locate and scan, ms[1] the block
 * decodes, ms[2] the answers; *touched_blocks (may be NULL) the blocks it
 * decoded.  With several decode waves, ms[1] also holds the answers of the
 * earlier waves.  Waits for the batch to finish. */
int tbg_probe_phase_ms(int handle, float ms[3], uint64_t *touched_blocks);

/* Device bytes of decoded-symbol scratch a grouped probe may hold (default
 * 16 GiB).  A touched block takes 16 KiB (codes of at most 256 emitted
 * symbols) or 32 KiB; blocks beyond the budget are decoded in further
 * waves.  No counterpart in the reference, which decodes per position. */
int tbg_probe_tune(uint64_t scratch_bytes);

/* encode_piece (probe.c:696) after list_squares (probe.c:1511) for n
 * queries: table index and table side (dev_side may be NULL). */
int tbg_encode_batch(int handle, const void *dev_queries, uint64_t n, uint64_t *dev_idx,
                     uint8_t *dev_side);

/* decode_piece (probe.c:1022) for the table's PIECE_ENC layout: the squares,
 * in table piece order (8 bytes per index), of the positions at indices
 * dev_idx[] of side `side`. */
int tbg_decode_batch(int handle, int side, const uint64_t *dev_idx, uint64_t n,
                     uint8_t *dev_squares);

/* n seeded random legal positions of a material (distinct squares, side
 * not to move not in check) as queries.  *failed counts queries for which
 * 64 draws found no legal position (their squares are the last draw). */
int tbg_gen_positions(const char *material, uint64_t seed, uint64_t n, void *dev_queries,
                      uint32_t *failed);

/* calc_sub_worker (tb8gen.c:280-314) for slice s with the 7-piece values
 * taken from the tables of the capture materials instead of the seeded
 * stub: handles[k] is an open table (tbg_probe_open) of the material left
 * when one piece of set k is captured (tbg_capture_material names it; only
 * the sets of colour stm are used).  mode 0 probes the tables (grouped rANS
 * decode on the GPU); mode 1 evaluates the tables' defining formula with
 * (seed, modulus) -- the values tbg_table_build stores -- without reading
 * them (handles may be NULL).  Both give the same bitmaps.  Outputs as for
 * tbg_calc_sub. */
int tbg_calc_sub_table(int stm, int s, void *const dev_cls[5], const int handles[6], int mode,
                       uint64_t seed, int modulus);

/* The material left when one piece of set `set` of the current material is
 * captured, as a name ("KRRvKRRR"), the material of the table that
 * tbg_calc_sub_table needs for that set. */
int tbg_capture_material(int set, char *name, int len);

/* ---- synthetic inputs (no counterpart in the reference) -------------- */

/* Seeded Bernoulli bitmap: bit i < nbits set iff the (i+1)-th output of the
 * splitmix64 stream keyed by (seed, tag) is below thr (P = thr / 2^64);
 * the rest of the `bytes` buffer is zeroed. */
int tbg_gen_bernoulli(void *dev, uint64_t nbits, uint64_t bytes, uint64_t seed,
                      uint64_t tag, uint64_t thr);

/* Reads n attack sets into out[] for squares sq[] and occupancies occ[]
 * (piece type 2..6 = N, B, R, Q, K): a test hook that checks the device
 * attack functions against movegen.h / magic.h. */
int tbg_attacks(int type, const uint8_t *dev_sq, const uint64_t *dev_occ,
                uint64_t *dev_out, uint64_t n);

#ifdef __cplusplus
}
#endif

#endif /* TBGPU_H */
