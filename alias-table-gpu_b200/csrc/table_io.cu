// table_io.cu — table files and the sharding of a batch of tables over devices (host code).
//
// Table file (little endian): a 64-byte header, the CSR offsets of the batch (num_tables + 1
// int64; a single table is one table), then n rows of {f32 prob, u32 alias}:
//   bytes  0.. 7  magic "WRSTABLE"
//          8..11  format version (1)
//         12..15  row bytes (8)
//         16..23  n (int64, rows)
//         24..31  num_tables (int64)
//         32..39  W (double: the weight total of a single table; 0 for a batch)
//         40..47  FNV-1a 64 of the offsets and rows
//         48..63  zero
// The reference keeps its tables in memory only (TableStorage.cuh:6-128); these files let a
// table built once be sampled later, by another process or on another device.
//
// Sharding: tables are independent, so a batch spreads over devices by contiguous table
// ranges with no exchange between them; wrs_shard_tables balances the ranges by items plus a
// per-table cost (a table of a few items still takes a launch slot and a header).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "host_util.h"

namespace {

constexpr char kMagic[8] = {'W', 'R', 'S', 'T', 'A', 'B', 'L', 'E'};
constexpr uint32_t kVersion = 1;
constexpr size_t kChunkRows = (size_t)1 << 22;  // 32 MiB of rows per transfer

struct FileHeader {
    char magic[8];
    uint32_t version;
    uint32_t row_bytes;
    int64_t n;
    int64_t num_tables;
    double W;
    uint64_t checksum;
    uint64_t pad[2];
};
static_assert(sizeof(FileHeader) == 64, "file header");

uint64_t fnv1a(uint64_t h, const void* p, size_t len) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < len; ++i) {
        h ^= b[i];
        h *= 0x100000001b3ull;
    }
    return h;
}
constexpr uint64_t kFnvBasis = 0xcbf29ce484222325ull;

bool offsets_valid(const int64_t* off, int64_t num_tables, int64_t n) {
    if (off[0] != 0 || off[num_tables] != n) return false;
    for (int64_t t = 0; t < num_tables; ++t)
        if (off[t + 1] < off[t]) return false;
    return true;
}

wrs_status write_file(const char* path, const wrs_alias_row* d_table, int64_t n, const int64_t* h_offsets,
                      int64_t num_tables, double W, cudaStream_t stream) {
    std::vector<int64_t> off(num_tables + 1);
    if (h_offsets) {
        std::memcpy(off.data(), h_offsets, sizeof(int64_t) * (num_tables + 1));
        if (!offsets_valid(off.data(), num_tables, n)) return WRS_ERR_INVALID_ARGUMENT;
    } else {
        off[0] = 0;
        off[1] = n;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return WRS_ERR_INVALID_ARGUMENT;
    FileHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.row_bytes = sizeof(wrs_alias_row);
    h.n = n;
    h.num_tables = num_tables;
    h.W = h_offsets ? 0.0 : W;
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    uint64_t sum = fnv1a(kFnvBasis, off.data(), sizeof(int64_t) * off.size());
    ok = ok && std::fwrite(off.data(), sizeof(int64_t), off.size(), f) == off.size();
    std::vector<wrs_alias_row> buf(std::min<size_t>((size_t)n, kChunkRows));
    wrs_status st = WRS_SUCCESS;
    for (int64_t r = 0; ok && r < n; r += (int64_t)buf.size()) {
        const size_t cnt = (size_t)std::min<int64_t>((int64_t)buf.size(), n - r);
        if (cudaMemcpyAsync(buf.data(), d_table + r, cnt * sizeof(wrs_alias_row), cudaMemcpyDeviceToHost, stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            st = WRS_ERR_CUDA;
            break;
        }
        sum = fnv1a(sum, buf.data(), cnt * sizeof(wrs_alias_row));
        ok = std::fwrite(buf.data(), sizeof(wrs_alias_row), cnt, f) == cnt;
    }
    if (ok && st == WRS_SUCCESS) {
        h.checksum = sum;
        ok = std::fseek(f, 0, SEEK_SET) == 0 && std::fwrite(&h, sizeof(h), 1, f) == 1;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (st != WRS_SUCCESS) return st;
    return ok ? WRS_SUCCESS : WRS_ERR_INVALID_ARGUMENT;
}

wrs_status read_header(FILE* f, FileHeader* h) {
    if (std::fread(h, sizeof(*h), 1, f) != 1) return WRS_ERR_INVALID_ARGUMENT;
    if (std::memcmp(h->magic, kMagic, 8) != 0 || h->version != kVersion || h->row_bytes != sizeof(wrs_alias_row) ||
        h->n < 1 || h->num_tables < 1 || h->num_tables > h->n + 1)
        return WRS_ERR_INVALID_ARGUMENT;
    return WRS_SUCCESS;
}

}  // namespace

extern "C" wrs_status wrs_table_file_write(const char* path, const wrs_alias_row* d_table, int64_t n, double W,
                                           void* stream) {
    if (!path || !d_table || n < 1) return WRS_ERR_INVALID_ARGUMENT;
    return write_file(path, d_table, n, nullptr, 1, W, static_cast<cudaStream_t>(stream));
}

extern "C" wrs_status wrs_batched_table_file_write(const char* path, const wrs_alias_row* d_table,
                                                   const int64_t* h_offsets, int64_t num_tables, void* stream) {
    if (!path || !d_table || !h_offsets || num_tables < 1) return WRS_ERR_INVALID_ARGUMENT;
    const int64_t n = h_offsets[num_tables];
    if (n < 1) return WRS_ERR_INVALID_ARGUMENT;
    return write_file(path, d_table, n, h_offsets, num_tables, 0.0, static_cast<cudaStream_t>(stream));
}

extern "C" wrs_status wrs_table_file_info(const char* path, int64_t* n, int64_t* num_tables, double* W) {
    if (!path) return WRS_ERR_INVALID_ARGUMENT;
    FILE* f = std::fopen(path, "rb");
    if (!f) return WRS_ERR_INVALID_ARGUMENT;
    FileHeader h;
    const wrs_status st = read_header(f, &h);
    std::fclose(f);
    if (st != WRS_SUCCESS) return st;
    if (n) *n = h.n;
    if (num_tables) *num_tables = h.num_tables;
    if (W) *W = h.W;
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_table_file_read(const char* path, wrs_alias_row* d_table, int64_t n,
                                          int64_t* h_offsets, int64_t num_tables, void* stream_) {
    if (!path || !d_table || n < 1 || num_tables < 1) return WRS_ERR_INVALID_ARGUMENT;
    FILE* f = std::fopen(path, "rb");
    if (!f) return WRS_ERR_INVALID_ARGUMENT;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    FileHeader h;
    wrs_status st = read_header(f, &h);
    if (st == WRS_SUCCESS && (h.n != n || h.num_tables != num_tables)) st = WRS_ERR_CAPACITY;
    std::vector<int64_t> off(num_tables + 1);
    if (st == WRS_SUCCESS &&
        (std::fread(off.data(), sizeof(int64_t), off.size(), f) != off.size() || !offsets_valid(off.data(), num_tables, n)))
        st = WRS_ERR_INVALID_ARGUMENT;
    uint64_t sum = fnv1a(kFnvBasis, off.data(), sizeof(int64_t) * off.size());
    std::vector<wrs_alias_row> buf(std::min<size_t>((size_t)n, kChunkRows));
    for (int64_t r = 0; st == WRS_SUCCESS && r < n; r += (int64_t)buf.size()) {
        const size_t cnt = (size_t)std::min<int64_t>((int64_t)buf.size(), n - r);
        if (std::fread(buf.data(), sizeof(wrs_alias_row), cnt, f) != cnt) {
            st = WRS_ERR_INVALID_ARGUMENT;
            break;
        }
        sum = fnv1a(sum, buf.data(), cnt * sizeof(wrs_alias_row));
        if (cudaMemcpyAsync(d_table + r, buf.data(), cnt * sizeof(wrs_alias_row), cudaMemcpyHostToDevice, stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            st = WRS_ERR_CUDA;
    }
    std::fclose(f);
    if (st == WRS_SUCCESS && sum != h.checksum) st = WRS_ERR_INVALID_ARGUMENT;
    if (st == WRS_SUCCESS && h_offsets) std::memcpy(h_offsets, off.data(), sizeof(int64_t) * off.size());
    return st;
}

extern "C" wrs_status wrs_shard_tables(const int64_t* h_offsets, int64_t num_tables, int32_t num_shards,
                                       int64_t table_cost, int64_t* h_bounds) {
    if (!h_offsets || !h_bounds || num_tables < 0 || num_shards < 1 || table_cost < 0) return WRS_ERR_INVALID_ARGUMENT;
    if (h_offsets[0] != 0) return WRS_ERR_INVALID_ARGUMENT;
    for (int64_t t = 0; t < num_tables; ++t)
        if (h_offsets[t + 1] < h_offsets[t]) return WRS_ERR_INVALID_ARGUMENT;
    // cost of tables [0, t): items + t * table_cost; shard s ends at the first table boundary
    // whose cost reaches s / num_shards of the total
    const double total = (double)h_offsets[num_tables] + (double)num_tables * (double)table_cost;
    h_bounds[0] = 0;
    int64_t t = 0;
    for (int32_t s = 1; s < num_shards; ++s) {
        const double target = total * s / num_shards;
        while (t < num_tables && (double)h_offsets[t] + (double)t * (double)table_cost < target) ++t;
        h_bounds[s] = t;
    }
    h_bounds[num_shards] = num_tables;
    for (int32_t s = 1; s <= num_shards; ++s)
        if (h_bounds[s] < h_bounds[s - 1]) h_bounds[s] = h_bounds[s - 1];
    return WRS_SUCCESS;
}
