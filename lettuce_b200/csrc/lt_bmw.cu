// Configuration files in the BMW format of the reference (IO/config_io/bmw_format.hpp):
// SaveConfigBMW / LoadConfigBMW (first two rows, header "#BMW") and SaveConfigBMWFull /
// LoadConfigBMWFull (all three rows, header "#18BMW").  The device packs the links into the
// file's big-endian record order and computes the Adler-64 checksum in the same pass
// (k_bmw_pack / k_bmw_unpack); the host only moves bytes and writes the 4096-byte header.
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lt_handle.h"
#include "lt_kernels.cuh"

namespace {

constexpr size_t kHeaderBytes = 4096;   // bmw_format.hpp:29-33

int check_h(const lt_lattice* h, const char* fn)
{
    if (!h) return lt::set_error(LT_ERR_ARG, (std::string(fn) + ": null handle").c_str());
    return LT_OK;
}

int launched(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return lt::cuda_error(e, what);
    return LT_OK;
}

size_t payload_bytes(const lt_lattice* h, int full) { return (size_t)h->g.V * 4 * (full ? 18 : 12) * sizeof(double); }

// The handle's host-transfer staging buffer (4V * 18 doubles) holds either payload
int staging(lt_lattice* h)
{
    if (h->d_aos) return LT_OK;
    LT_CK(cudaSetDevice(h->device));
    LT_CK(cudaMalloc((void**)&h->d_aos, (size_t)4 * h->g.V * 18 * sizeof(double)));
    return LT_OK;
}

// Checksum_Adler64::Finalize (bmw_format.hpp:89-96) of the per-block partial sums
int finish_checksum(lt_lattice* h, const unsigned long long* d_partials, uint64_t* out)
{
    std::vector<unsigned long long> p(2 * lt::kRedBlocks);
    LT_CK(cudaMemcpyAsync(p.data(), d_partials, sizeof(unsigned long long) * p.size(), cudaMemcpyDeviceToHost,
                          h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    uint64_t A = 0, B = 0;
    for (int k = 0; k < lt::kRedBlocks; ++k)
    {
        A = (A + p[k]) % lt::kAdler64Prime;
        B = (B + p[lt::kRedBlocks + k]) % lt::kAdler64Prime;
    }
    *out = ((B % lt::kAdler64Prime) << 32) + (A + 1) % lt::kAdler64Prime;
    return LT_OK;
}

// Checksum_Adler64::ReturnString (bmw_format.hpp:99-113): lower-case hex without padding
std::string hex(uint64_t v)
{
    char s[32];
    std::snprintf(s, sizeof(s), "%" PRIx64, v);
    return s;
}

int pack(lt_lattice* h, int full, bool to_staging, uint64_t* checksum)
{
    if (to_staging) LT_TRY(staging(h));
    auto* partials = reinterpret_cast<unsigned long long*>(h->partials);
    h->be->bmw_pack(h->ctx(), h->U, full, to_staging ? h->d_aos : nullptr, partials);
    LT_TRY(launched("bmw pack"));
    return finish_checksum(h, partials, checksum);
}

struct File
{
    std::FILE* f = nullptr;
    ~File()
    {
        if (f) std::fclose(f);
    }
};

} // namespace

extern "C" {

int lt_bmw_checksum(lt_lattice* h, int full, uint64_t* checksum)
{
    LT_TRY(check_h(h, "lt_bmw_checksum"));
    const lt::DeviceScope device_scope(h->device);
    if (!checksum) return lt::set_error(LT_ERR_ARG, "lt_bmw_checksum: null pointer");
    return pack(h, full ? 1 : 0, false, checksum);
}

int lt_save_bmw(lt_lattice* h, const char* path, int full, int overwrite, char* checksum_hex)
{
    LT_TRY(check_h(h, "lt_save_bmw"));
    const lt::DeviceScope device_scope(h->device);
    if (!path) return lt::set_error(LT_ERR_ARG, "lt_save_bmw: null path");
    full = full ? 1 : 0;
    if (!overwrite)
    {
        std::FILE* probe = std::fopen(path, "rb");
        if (probe)
        {
            std::fclose(probe);
            return lt::set_error(LT_ERR_IO, (std::string("lt_save_bmw: ") + path + " exists").c_str());
        }
    }
    uint64_t ck = 0;
    LT_TRY(pack(h, full, true, &ck));
    const std::string cks = hex(ck);
    // header (bmw_format.hpp:346-363): "#BMW Nx Ny Nz Nt <checksum>\n" then "\nGenerated with
    // Lettuce\n" and its terminating NUL, the rest of the 4096 bytes filled with '\n'
    std::vector<char> header(kHeaderBytes, '\n');
    const int n = std::snprintf(header.data(), kHeaderBytes, "%s %d %d %d %d %s\n", full ? "#18BMW" : "#BMW", h->ext[1],
                                h->ext[2], h->ext[3], h->ext[0], cks.c_str());
    if (n < 0 || (size_t)n >= kHeaderBytes) return lt::set_error(LT_ERR_IO, "lt_save_bmw: header too long");
    const int m = std::snprintf(header.data() + n, kHeaderBytes - (size_t)n, "\nGenerated with Lettuce\n");
    if (m < 0 || (size_t)(n + m) >= kHeaderBytes) return lt::set_error(LT_ERR_IO, "lt_save_bmw: header too long");
    const size_t bytes = payload_bytes(h, full);
    std::vector<unsigned char> payload(bytes);
    LT_CK(cudaMemcpyAsync(payload.data(), h->d_aos, bytes, cudaMemcpyDeviceToHost, h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    File file;
    file.f = std::fopen(path, "wb");
    if (!file.f) return lt::set_error(LT_ERR_IO, (std::string("lt_save_bmw: cannot open ") + path).c_str());
    if (std::fwrite(header.data(), 1, kHeaderBytes, file.f) != kHeaderBytes ||
        std::fwrite(payload.data(), 1, bytes, file.f) != bytes)
        return lt::set_error(LT_ERR_IO, (std::string("lt_save_bmw: write failed on ") + path).c_str());
    const int closed = std::fclose(file.f);
    file.f = nullptr;
    if (closed != 0) return lt::set_error(LT_ERR_IO, (std::string("lt_save_bmw: close failed on ") + path).c_str());
    if (checksum_hex) std::snprintf(checksum_hex, 17, "%s", cks.c_str());
    return LT_OK;
}

int lt_load_bmw(lt_lattice* h, const char* path, int full, int* checksum_ok, int* in_group)
{
    LT_TRY(check_h(h, "lt_load_bmw"));
    const lt::DeviceScope device_scope(h->device);
    if (!path) return lt::set_error(LT_ERR_ARG, "lt_load_bmw: null path");
    full = full ? 1 : 0;
    File file;
    file.f = std::fopen(path, "rb");
    if (!file.f) return lt::set_error(LT_ERR_IO, (std::string("lt_load_bmw: cannot open ") + path).c_str());
    // header (bmw_format.hpp:185-205): "#BMW Nx Ny Nz Nt checksum" (or "#18BMW ...")
    std::vector<char> header(kHeaderBytes + 1, '\0');
    if (std::fread(header.data(), 1, kHeaderBytes, file.f) != kHeaderBytes)
        return lt::set_error(LT_ERR_IO, "lt_load_bmw: short header");
    int nx = 0, ny = 0, nz = 0, nt = 0;
    char ck_read[32] = { 0 };
    const int got = std::sscanf(header.data(), full ? "#18BMW %d %d %d %d %31s" : "#BMW %d %d %d %d %31s", &nx, &ny,
                                &nz, &nt, ck_read);
    if (got < 5) return lt::set_error(LT_ERR_IO, "lt_load_bmw: header does not match the expected format");
    if (nx != h->ext[1] || ny != h->ext[2] || nz != h->ext[3] || nt != h->ext[0])
        return lt::set_error(LT_ERR_ARG, "lt_load_bmw: lattice shape in the file differs from the handle's");
    const size_t bytes = payload_bytes(h, full);
    std::vector<unsigned char> payload(bytes);
    if (std::fread(payload.data(), 1, bytes, file.f) != bytes)
        return lt::set_error(LT_ERR_IO, "lt_load_bmw: file shorter than its lattice");
    LT_TRY(staging(h));
    LT_CK(cudaMemcpyAsync(h->d_aos, payload.data(), bytes, cudaMemcpyHostToDevice, h->stream));
    unsigned* flags = h->status + 2;
    LT_CK(cudaMemsetAsync(flags, 0, sizeof(unsigned), h->stream));
    auto* partials = reinterpret_cast<unsigned long long*>(h->partials);
    h->be->bmw_unpack(h->ctx(), h->U, full, h->d_aos, partials, flags);
    LT_TRY(launched("lt_load_bmw"));
    uint64_t ck = 0;
    LT_TRY(finish_checksum(h, partials, &ck));
    unsigned fl = 0;
    LT_CK(cudaMemcpyAsync(&fl, flags, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    if (checksum_ok) *checksum_ok = hex(ck) == std::string(ck_read) ? 1 : 0;
    if (in_group) *in_group = (fl & 1u) ? 0 : 1;
    return LT_OK;
}

} // extern "C"
