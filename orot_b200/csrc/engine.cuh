// engine.cuh -- data layout shared by the host planner and the sm_100a kernels.
//
// Work is described by three tables that live in HBM:
//   Stream  : one compressed output (raw / zlib / gzip framing + trailer).
//   Segment : a contiguous input range with its own LZ77 dictionary; it
//             becomes exactly one DEFLATE block (the whole buffer for
//             deflate_compress, one chunk for deflate_parallel_compress,
//             src/compress/block_compressor.cpp:16-73 and
//             src/parallel/parallel_compressor.cpp:65-84).
//   Tile    : at most tile_size bytes of one segment, the unit one warp walks.
//             Tiles of the same segment run concurrently: each starts with the
//             hash-table state carried in from earlier tiles and parses from
//             its own start; a sequential pass then moves the parse entry to
//             where the previous tile's parse really ended.
#pragma once
#include <cstdint>

namespace orotb {

constexpr int kFmtRaw = 0, kFmtZlib = 1, kFmtGzip = 2;
constexpr int kBlkStored = 0, kBlkFixed = 1, kBlkDynamic = 2;

// Segment flags.
constexpr uint32_t kSegLast = 1u;        // BFINAL block of its stream
constexpr uint32_t kSegWholeBuf = 2u;    // whole-buffer rule: all-literal parse -> stored
constexpr uint32_t kSegFault = 8u;       // set by a kernel that could not finish the segment (its stream fails)

// Stream error codes written to Stream::error.
constexpr uint32_t kErrNone = 0, kErrCapacity = 1, kErrInternal = 2;

struct Stream {
  uint64_t in_off;     // byte offset of the input in the input arena
  uint64_t in_len;
  uint64_t out_off;    // byte offset of the output slot (16-byte aligned)
  uint64_t out_cap;    // caller capacity for the whole framed stream
  uint32_t seg_first, seg_count;
  uint32_t piece_first, piece_count;
  int32_t level;       // unclamped caller level (gzip XFL uses it)
  uint32_t fmt;
  uint32_t parallel;   // 1: pigz framing (gzip XFL = 0)
  uint32_t ck_first, ck_count;  // checksum blocks of this stream
  uint32_t mode;       // kStreamBare | kStreamOpen
  uint32_t pad2;
  // results
  uint64_t out_size;   // framed bytes, 0 on error
  uint64_t raw_bits;   // bits of the raw DEFLATE part
  uint32_t checksum;
  uint32_t error;
};
// Stream modes for one rank's part of a stream compressed across GPUs:
// Bare: no header or trailer (the checksum of fmt is still computed);
// Open: another part follows, so no block is BFINAL and the part ends with an
// empty stored block, a sync point that leaves it on a byte boundary.
constexpr uint32_t kStreamBare = 1u, kStreamOpen = 2u;

struct Segment {
  uint64_t in_off;     // absolute byte offset in the input arena
  uint32_t len;
  uint32_t stream;
  uint32_t tile_first, tile_count;
  uint32_t flags;
  int32_t level;       // clamped 0..12
  // levels 4+: code table (288 litlen + 32 distance entries, code | len << 16),
  // header bits (HLIT..code lengths) and end-of-block code
  uint64_t codes;      // scratch byte offset of the code table
  uint64_t hdr_off;    // scratch byte offset of the HLIT..code-lengths bits
  uint32_t hdr_bits;
  uint32_t eob;        // EOB code | (code length << 16)
  // filled by the planner kernel
  uint32_t block_type;
  uint32_t piece_off;  // first copy slot of this block, from the stream's piece_first
  uint64_t bit_off;    // block start, in bits from the stream's raw start
  uint64_t bits;       // block length in bits (stored: for its actual offset)
};

// Per-window parse record of a speculative tile walk (32 input positions).
struct WinRec {
  uint32_t entry;      // first parse position >= window start (tile-relative)
  uint32_t bit;        // bit offset of that token in the tile's stream
  uint32_t matches;    // match tokens before it
  uint32_t run;        // D when all 32 positions have candidate distance D <= 32
                       // and equal the bytes D earlier (a run window), else 0;
                       // in the fast-level kernels' records, bits 8.. hold the
                       // first window after the run
};

struct Tile {
  uint32_t seg;
  uint32_t start;      // segment-relative
  uint32_t len;
  uint32_t index;      // index within the segment
  uint64_t scratch;    // byte offset of this tile's bit buffers in the scratch arena
  uint64_t rec;        // byte offset of WinRec[] (tiles with index > 0)
  uint64_t carry;      // byte offset of the carried-in hash table (index > 0)
  uint64_t slot;       // byte offset of this tile's published table (index < count-1)
  uint64_t cand;       // levels 1-3, index > 0: u16 per position, candidate distance
                       // that passed the first-byte check (0 = literal)
  uint64_t tok;        // levels 4+: token word per position (0 = not a match start)
  uint64_t hist;       // levels 4+: 320-bin literal/length + distance histogram
  // speculative walk (entry = tile start)
  uint32_t spec_bits, spec_matches, spec_exit, spec_tokens;
  // resolved parse: piece A = fix-up bits [0, fix_bits) from the fix-up
  // buffer, piece B = speculative bits [splice_bit, spec_bits)
  uint32_t fix_bits, splice_bit, fin_matches, fin_exit;
  uint32_t fix_entry;  // parse entry the fix-up assumed
  uint32_t pad1;
};

// A bit-range copy for the join kernel.  src == nullptr means "write the
// low nbits of value".
struct Piece {
  const uint32_t* src;  // 4-byte aligned source words
  uint32_t* dst;        // the stream's output slot (16-byte aligned)
  uint64_t src_bit;     // first bit within src
  uint64_t dst_bit;     // first bit within dst
  uint32_t nbits;
  uint32_t value;
};

// Checksum block: a range of one stream's input.
struct CkBlock {
  uint64_t in_off;     // absolute
  uint32_t len;
  uint32_t stream;
  uint32_t crc;        // raw CRC register from 0 (no conditioning)
  uint32_t a, b;       // Adler partial sums mod 65521
  uint32_t what;       // kCkCrc | kCkAdler: the sums the stream needs
};
constexpr uint32_t kCkCrc = 1u, kCkAdler = 2u;

// Limits.
constexpr int kMaxTileLog2 = 16;           // 64 KiB tiles at most
constexpr int kWindow = 32;

__host__ __device__ inline uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

// Worst case bits of a tile's fixed-Huffman token stream: a literal costs at
// most 9 bits and a match at most 25 bits per 3 covered bytes, so 9 bits per
// input byte plus one match (31 bits) hanging over the tile end.
__host__ __device__ inline uint64_t tile_stream_bytes(uint32_t tile_len) { return align_up(uint64_t(tile_len) * 9 / 8 + 64, 128); }

// Levels 4+ use dynamic codes of up to 15 bits: a literal costs at most 15
// bits and a match at most 48 bits per 3 covered bytes (16 bits per byte).
__host__ __device__ inline uint64_t lazy_stream_bytes(uint32_t tile_len) { return align_up(uint64_t(tile_len) * 2 + 256, 128); }

// Levels 4+: tiles of 16 x 258 bytes, each searching a 32 KiB window before
// it.  A multiple of the longest match keeps runs of 258-byte matches (zero
// fill, short periods) aligned with tile boundaries, so cutting the input
// into independent tiles costs no extra token on such data.  One CTA walks a
// run of kLazyRun consecutive tiles, sliding its window.
constexpr uint32_t kLazyTile = 16 * 258;
constexpr uint32_t kLazyRun = 32;
constexpr uint32_t kLazyWindow = 32768;

}  // namespace orotb
