// RSDFT's wavefunction file (wf.dat1), written and read for one process.
//
// Format (simple_wf_io_write, io_write_module.f90:19-264; read back by
// simple_wf_io_read, io_read_module.f90:15-521): Fortran sequential
// unformatted records, each framed by a 4-byte little-endian length marker
// before and after it (the default of the Fortran compilers RSDFT builds
// with; records above 2^31 - 9 bytes, which need split records, are
// refused).  New format (OC < 10):
//   -1 | ML, ML1, ML2, ML3 | MB, MBwr1, MBwr2 | MK, MS, MMBZ |
//   IO_ctrl, OC, TYPE_WF | LL2(3, ML) | occ(MB, MK, MS) | aa, bb, kbb(3, MMBZ) |
//   np(0:7) | grid id, ir | band id, ir | bzsm id, ir | spin id, ir |
//   then unk(:, n, k, s) for s = 1..MS, k = 1..MK, n = MBwr1..MBwr2,
//   real(8) or, for OC = 4 and 5, real(4).
// Old format (OC >= 10): ML.. | MB.. | LL2 | occ | bands (real(8)).
// TYPE_WF = 1 marks real (Gamma) data.  With one process the layout records
// are np = 1 and id = 0, ir = the full count in each dimension, and LL2 lists
// the grid points x fastest (SYStype = 0 over the whole grid).
//
// Device-resident arrays (a registered host array's mirror, or device
// memory) move band by band through two pinned buffers: the copy of the
// next band runs while the current one is written (or, reading, the copy of
// the current band while the next one is read).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace rsdft {
namespace {

constexpr size_t kMaxRecord = 2147483639;  // one pair of 4-byte markers

struct File {
    FILE* f = nullptr;
    std::vector<char> vbuf;
    std::string path;
    ~File() {
        if (f) fclose(f);
    }
    int open(const std::string& p, const char* mode) {
        path = p;
        f = fopen(p.c_str(), mode);
        if (!f) {
            set_error("cannot open '%s' (mode %s)", p.c_str(), mode);
            return RSDFT_EINVAL;
        }
        vbuf.resize((size_t)8 << 20);
        setvbuf(f, vbuf.data(), _IOFBF, vbuf.size());
        return RSDFT_OK;
    }
    int close() {
        const int rc = fclose(f);
        f = nullptr;
        if (rc != 0) {
            set_error("error closing '%s'", path.c_str());
            return RSDFT_EINVAL;
        }
        return RSDFT_OK;
    }
};

struct Part {
    const void* p;
    size_t n;
};

int write_record(File& fh, std::initializer_list<Part> parts) {
    size_t len = 0;
    for (const Part& q : parts) len += q.n;
    if (len > kMaxRecord) {
        set_error("'%s': record of %zu bytes exceeds one 4-byte-marker record", fh.path.c_str(), len);
        return RSDFT_EUNSUP;
    }
    const int32_t m = (int32_t)len;
    bool ok = fwrite(&m, 4, 1, fh.f) == 1;
    for (const Part& q : parts) ok = ok && (q.n == 0 || fwrite(q.p, 1, q.n, fh.f) == q.n);
    ok = ok && fwrite(&m, 4, 1, fh.f) == 1;
    if (!ok) {
        set_error("write to '%s' failed", fh.path.c_str());
        return RSDFT_EINVAL;
    }
    return RSDFT_OK;
}

template <typename T>
int write_values(File& fh, const std::vector<T>& v) {
    return write_record(fh, {{v.data(), v.size() * sizeof(T)}});
}

// Leading marker of the next record; *len = its length in bytes.
int record_head(File& fh, size_t* len, const char* what) {
    int32_t m = 0;
    if (fread(&m, 4, 1, fh.f) != 1) {
        set_error("'%s': file ends before the %s record", fh.path.c_str(), what);
        return RSDFT_EINVAL;
    }
    if (m < 0) {
        set_error("'%s': the %s record is split (over 2 GiB); not supported", fh.path.c_str(), what);
        return RSDFT_EUNSUP;
    }
    *len = (size_t)m;
    return RSDFT_OK;
}

int record_tail(File& fh, size_t len, const char* what) {
    int32_t m = 0;
    if (fread(&m, 4, 1, fh.f) != 1 || (size_t)m != len) {
        set_error("'%s': bad length marker after the %s record", fh.path.c_str(), what);
        return RSDFT_EINVAL;
    }
    return RSDFT_OK;
}

// Read a record of at least `bytes` bytes into dst (a Fortran read may take
// fewer items than the record holds; the rest is skipped).
int read_record(File& fh, void* dst, size_t bytes, const char* what) {
    size_t len = 0;
    RS_CHECK(record_head(fh, &len, what));
    if (len < bytes) {
        set_error("'%s': the %s record holds %zu bytes, %zu expected", fh.path.c_str(), what, len, bytes);
        return RSDFT_EINVAL;
    }
    if (bytes && fread(dst, 1, bytes, fh.f) != bytes) {
        set_error("'%s': file ends inside the %s record", fh.path.c_str(), what);
        return RSDFT_EINVAL;
    }
    if (len > bytes && fseek(fh.f, (long)(len - bytes), SEEK_CUR) != 0) {
        set_error("'%s': seek failed in the %s record", fh.path.c_str(), what);
        return RSDFT_EINVAL;
    }
    return record_tail(fh, len, what);
}

int skip_record(File& fh, const char* what) { return read_record(fh, nullptr, 0, what); }

// Where the bands live: a host array, or device memory (a registered array's
// mirror, or a device pointer), moved through two pinned band buffers.
struct Bands {
    double* host = nullptr;  // plain host array
    double* dev = nullptr;   // device-resident
    double* pin[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~Bands() {
        for (int i = 0; i < 2; ++i) {
            if (pin[i]) cudaFreeHost(pin[i]);
            if (ev[i]) cudaEventDestroy(ev[i]);
        }
    }
};

// Resolve unk; for device-resident data check the extent against a
// registration and set up the pinned buffers.
int bands_open(Bands& b, const double* unk, size_t span, long ml) {
    void* d = nullptr;
    const int r = resolve(unk, span * sizeof(double), &d);
    if (r < 0) return r;
    if (!r) {
        b.host = const_cast<double*>(unk);
        return RSDFT_OK;
    }
    RS_CHECK(require_init());
    b.dev = static_cast<double*>(d);
    for (int i = 0; i < 2; ++i) {
        RS_CUDA(cudaMallocHost(&b.pin[i], sizeof(double) * (size_t)ml));
        RS_CUDA(cudaEventCreateWithFlags(&b.ev[i], cudaEventDisableTiming));
    }
    return RSDFT_OK;
}

bool oc_single(int oc) { return oc == 4 || oc == 5; }

std::string split_name(const char* path) { return std::string(path) + ".00000"; }

}  // namespace
}  // namespace rsdft

using namespace rsdft;

extern "C" int rsdft_gpu_write_wf(const char* path, const double* unk, long ld, int mb, int mk, int ms, int mbwr1,
                                  int mbwr2, int oc, int io_ctrl, const int* ngrid, const double* occ,
                                  const double* aa, const double* bb, int mmbz, const double* kbb) {
    RS_ENTRY();
    if (!path || !unk || !ngrid || mb < 1 || mk < 1 || ms < 1 || mmbz < 0) {
        set_error("write_wf: NULL path/unk/ngrid or bad counts");
        return RSDFT_EINVAL;
    }
    if (io_ctrl != 0 && io_ctrl != 3) {
        set_error("write_wf: io_ctrl %d (only 0 and 3 are written)", io_ctrl);
        return RSDFT_EUNSUP;
    }
    const int n1 = ngrid[0], n2 = ngrid[1], n3 = ngrid[2];
    if (n1 < 1 || n2 < 1 || n3 < 1) {
        set_error("write_wf: bad grid %d x %d x %d", n1, n2, n3);
        return RSDFT_EINVAL;
    }
    const long ml = (long)n1 * n2 * n3;
    if (ld < ml) {
        set_error("write_wf: ld %ld < ML %ld", ld, ml);
        return RSDFT_EINVAL;
    }
    // the reference's own correction of the band range (io_write_module.f90:80-81)
    if (mbwr1 < 1 || mbwr2 < mbwr1 || mb < mbwr1) mbwr1 = 1;
    if (mbwr2 < 1 || mbwr2 < mbwr1 || mb < mbwr2) mbwr2 = mb;
    const bool single = oc_single(oc), oldfmt = oc >= 10;

    Bands b;
    const size_t span = (size_t)ld * ((size_t)mb * mk * ms - 1) + (size_t)ml;
    RS_CHECK(bands_open(b, unk, span, ml));

    File fh;
    RS_CHECK(fh.open(path, "wb"));
    // ---- header
    std::vector<int32_t> ll2((size_t)3 * ml);
    for (long i = 0; i < ml; ++i) {
        ll2[3 * i] = (int32_t)(i % n1);
        ll2[3 * i + 1] = (int32_t)((i / n1) % n2);
        ll2[3 * i + 2] = (int32_t)(i / ((long)n1 * n2));
    }
    std::vector<double> occv((size_t)mb * mk * ms, 0.0);
    if (occ) std::memcpy(occv.data(), occ, occv.size() * sizeof(double));
    const std::vector<int32_t> dims{(int32_t)ml, n1, n2, n3}, bands{mb, mbwr1, mbwr2};
    if (!oldfmt) {
        RS_CHECK(write_values(fh, std::vector<int32_t>{-1}));
        RS_CHECK(write_values(fh, dims));
        RS_CHECK(write_values(fh, bands));
        RS_CHECK(write_values(fh, std::vector<int32_t>{mk, ms, mmbz}));
        RS_CHECK(write_values(fh, std::vector<int32_t>{io_ctrl, oc, 1}));
        RS_CHECK(write_values(fh, ll2));
        RS_CHECK(write_values(fh, occv));
        std::vector<double> lat(18 + (size_t)3 * mmbz, 0.0);
        if (aa) std::memcpy(lat.data(), aa, 9 * sizeof(double));
        if (bb) std::memcpy(lat.data() + 9, bb, 9 * sizeof(double));
        if (kbb && mmbz > 0) std::memcpy(lat.data() + 18, kbb, (size_t)3 * mmbz * sizeof(double));
        RS_CHECK(write_values(fh, lat));
        RS_CHECK(write_values(fh, std::vector<int32_t>(8, 1)));  // np(0:7) of one process
        for (int32_t count : {(int32_t)ml, mb, mk, ms}) RS_CHECK(write_values(fh, std::vector<int32_t>{0, count}));
    } else {
        RS_CHECK(write_values(fh, dims));
        RS_CHECK(write_values(fh, bands));
        RS_CHECK(write_values(fh, ll2));
        RS_CHECK(write_values(fh, occv));
    }
    File split;
    File* out = &fh;
    if (io_ctrl == 3) {
        RS_CHECK(fh.close());
        RS_CHECK(split.open(split_name(path), "wb"));
        out = &split;
    }
    // ---- bands: s, k, n = mbwr1..mbwr2
    std::vector<long> offs;
    for (int s = 0; s < ms; ++s)
        for (int k = 0; k < mk; ++k)
            for (int n = mbwr1 - 1; n < mbwr2; ++n) offs.push_back(ld * ((long)n + (long)mb * (k + (long)mk * s)));
    std::vector<float> sp(single ? (size_t)ml : 0);
    cudaStream_t st = b.dev ? ctx().stream : nullptr;
    auto issue = [&](size_t i) -> int {
        RS_CUDA(cudaMemcpyAsync(b.pin[i & 1], b.dev + offs[i], sizeof(double) * (size_t)ml, cudaMemcpyDeviceToHost,
                                st));
        RS_CUDA(cudaEventRecord(b.ev[i & 1], st));
        return RSDFT_OK;
    };
    if (b.dev && !offs.empty()) RS_CHECK(issue(0));
    for (size_t i = 0; i < offs.size(); ++i) {
        const double* src = b.host ? b.host + offs[i] : b.pin[i & 1];
        if (b.dev) {
            RS_CUDA(cudaEventSynchronize(b.ev[i & 1]));
            if (i + 1 < offs.size()) RS_CHECK(issue(i + 1));  // into the buffer written out last round
        }
        if (single) {
            for (long j = 0; j < ml; ++j) sp[j] = (float)src[j];
            RS_CHECK(write_values(*out, sp));
        } else {
            RS_CHECK(write_record(*out, {{src, sizeof(double) * (size_t)ml}}));
        }
    }
    return out->close();
}

extern "C" int rsdft_gpu_read_wf(const char* path, double* unk, long ld, int mb, int mk, int ms, int io_ctrl,
                                 const int* ngrid, double* occ, int* info) {
    RS_ENTRY();
    if (!path || !unk || !ngrid || mb < 1 || mk < 1 || ms < 1) {
        set_error("read_wf: NULL path/unk/ngrid or bad counts");
        return RSDFT_EINVAL;
    }
    if (io_ctrl != 0 && io_ctrl != 3) {
        set_error("read_wf: io_ctrl %d (only 0 and 3 are read)", io_ctrl);
        return RSDFT_EUNSUP;
    }
    const int n1 = ngrid[0], n2 = ngrid[1], n3 = ngrid[2];
    if (n1 < 1 || n2 < 1 || n3 < 1) {
        set_error("read_wf: bad grid %d x %d x %d", n1, n2, n3);
        return RSDFT_EINVAL;
    }
    const long ml = (long)n1 * n2 * n3;
    if (ld < ml) {
        set_error("read_wf: ld %ld < ML %ld", ld, ml);
        return RSDFT_EINVAL;
    }
    File fh;
    RS_CHECK(fh.open(path, "rb"));
    // ---- header (io_read_module.f90:126-150)
    int32_t first = 0;
    size_t len = 0;
    RS_CHECK(record_head(fh, &len, "first"));
    const bool newfmt = len >= 4 && fread(&first, 4, 1, fh.f) == 1 && first < 0;
    if (newfmt) {
        if (len > 4) fseek(fh.f, (long)(len - 4), SEEK_CUR);
        RS_CHECK(record_tail(fh, len, "first"));
    } else {
        rewind(fh.f);
    }
    int32_t h[13] = {0};
    RS_CHECK(read_record(fh, h, 4 * sizeof(int32_t), "grid size"));
    RS_CHECK(read_record(fh, h + 4, 3 * sizeof(int32_t), "band range"));
    if (newfmt) {
        RS_CHECK(read_record(fh, h + 7, 3 * sizeof(int32_t), "k/spin count"));
        RS_CHECK(read_record(fh, h + 10, 3 * sizeof(int32_t), "io/precision flags"));
    } else {
        h[7] = mk;  // the old format has no k / spin counts: the caller's (io_read_module.f90:146-147)
        h[8] = ms;
    }
    if (info) std::memcpy(info, h, sizeof(h));
    if (h[0] != ml || h[1] != n1 || h[2] != n2 || h[3] != n3) {
        set_error("read_wf: file grid %d (%d x %d x %d), expected %ld (%d x %d x %d)", h[0], h[1], h[2], h[3], ml,
                  n1, n2, n3);
        return RSDFT_EINVAL;
    }
    const int fmb = h[4], fmb1 = h[5], fmb2 = h[6], fmk = h[7], fms = h[8], fmmbz = h[9], foc = h[11];
    if (fmb < 1 || fmb1 < 1 || fmb2 < fmb1 || fmk < 1 || fms < 1 || fmmbz < 0) {
        set_error("read_wf: bad counts in the header (MB %d, %d..%d, MK %d, MS %d)", fmb, fmb1, fmb2, fmk, fms);
        return RSDFT_EINVAL;
    }
    if (newfmt && h[12] != 1) {
        set_error("read_wf: TYPE_WF %d (complex data) in a real Gamma-point read", h[12]);
        return RSDFT_EUNSUP;
    }
    const bool single = newfmt && oc_single(foc);
    // ---- grid map: file point i -> grid index
    std::vector<int32_t> ll2((size_t)3 * ml);
    RS_CHECK(read_record(fh, ll2.data(), ll2.size() * sizeof(int32_t), "LL2"));
    std::vector<long> perm((size_t)ml);
    std::vector<char> seen((size_t)ml, 0);
    bool identity = true;
    for (long i = 0; i < ml; ++i) {
        const int a = ll2[3 * i], b2 = ll2[3 * i + 1], c = ll2[3 * i + 2];
        if (a < 0 || a >= n1 || b2 < 0 || b2 >= n2 || c < 0 || c >= n3) {
            set_error("read_wf: LL2 point %ld = (%d, %d, %d) outside the grid", i + 1, a, b2, c);
            return RSDFT_EINVAL;
        }
        const long j = a + (long)n1 * (b2 + (long)n2 * c);
        if (seen[j]++) {
            set_error("read_wf: LL2 lists grid point (%d, %d, %d) twice", a, b2, c);
            return RSDFT_EINVAL;
        }
        perm[i] = j;
        identity = identity && j == i;
    }
    // ---- occupations over the common ranges (io_read_module.f90:218-237)
    std::vector<double> focc((size_t)fmb * fmk * fms);
    RS_CHECK(read_record(fh, focc.data(), focc.size() * sizeof(double), "occ"));
    if (occ) {
        for (int s = 0; s < std::min(ms, fms); ++s)
            for (int k = 0; k < std::min(mk, fmk); ++k)
                for (int n = 0; n < std::min(mb, fmb); ++n)
                    occ[n + (long)mb * (k + (long)mk * s)] = focc[n + (long)fmb * (k + (long)fmk * s)];
    }
    if (newfmt) {
        RS_CHECK(skip_record(fh, "lattice"));
        for (const char* w : {"np", "grid layout", "band layout", "k layout", "spin layout"})
            RS_CHECK(skip_record(fh, w));
    }
    File split;
    File* in = &fh;
    if (io_ctrl == 3) {
        RS_CHECK(split.open(split_name(path), "rb"));
        in = &split;
    }
    // ---- bands
    Bands b;
    const size_t span = (size_t)ld * ((size_t)mb * mk * ms - 1) + (size_t)ml;
    RS_CHECK(bands_open(b, unk, span, ml));
    cudaStream_t st = b.dev ? ctx().stream : nullptr;
    std::vector<float> sp(single ? (size_t)ml : 0);
    std::vector<double> tmp(identity ? 0 : (size_t)ml);
    size_t used = 0;  // bands copied to the device so far (pinned buffer use count)
    for (int s = 0; s < fms; ++s)
        for (int k = 0; k < fmk; ++k)
            for (int n = fmb1 - 1; n < fmb2; ++n) {
                if (n >= mb || k >= mk || s >= ms) {
                    RS_CHECK(skip_record(*in, "band"));
                    continue;
                }
                const long off = ld * ((long)n + (long)mb * (k + (long)mk * s));
                double* dst = b.host ? b.host + off : b.pin[used & 1];
                if (b.dev && used >= 2) RS_CUDA(cudaEventSynchronize(b.ev[used & 1]));  // its last copy is done
                double* land = identity ? dst : tmp.data();
                if (single) {
                    RS_CHECK(read_record(*in, sp.data(), sp.size() * sizeof(float), "band"));
                    for (long j = 0; j < ml; ++j) land[j] = (double)sp[j];
                } else {
                    RS_CHECK(read_record(*in, land, sizeof(double) * (size_t)ml, "band"));
                }
                if (!identity)
                    for (long j = 0; j < ml; ++j) dst[perm[j]] = tmp[j];
                if (b.dev) {
                    RS_CUDA(cudaMemcpyAsync(b.dev + off, dst, sizeof(double) * (size_t)ml, cudaMemcpyHostToDevice, st));
                    RS_CUDA(cudaEventRecord(b.ev[used & 1], st));
                    ++used;
                }
            }
    if (b.dev) RS_CUDA(cudaStreamSynchronize(st));
    return RSDFT_OK;
}


// ----------------------------------------------------------------- vrho
// RSDFT's density/potential file (vrho.dat1), one process.  Format
// (write_data, io_module.f90:97-226; read back by read_data,
// io_module.f90:283-432), sequential unformatted records as above:
//   version (character(64) "version3.0, comment_length=64") |
//   ML, ML1, ML2, ML3 | LL2(3, ML) | comment | aa(3, 3) | comment |
//   Nelement, Natom | aa_atom(3, Natom) | ki_atom(Natom) | zn_atom(Nelement) |
//   comment | efermi |
//   then for s = 1..MSP: rho(:, s) | Vloc(:, s) | Vh (s = 1 only) | Vxc(:, s).
// Files without the version record (the reference's older writer) hold no
// comment, lattice, atom or Fermi records: the fields follow LL2.  The
// reader places each value by the file's LL2 map, so a file written under
// any grid-point order of the same grid reads back.

namespace rsdft {
namespace {

std::vector<char> text64(const char* s) {
    std::vector<char> t(64, ' ');
    std::memcpy(t.data(), s, std::min<size_t>(64, std::strlen(s)));
    return t;
}

// n doubles of a host array or of device memory (a registered array's
// mirror, or a device pointer) into v.
int fetch_field(const double* p, size_t n, std::vector<double>& v) {
    void* d = nullptr;
    const int r = resolve(p, n * sizeof(double), &d);
    if (r < 0) return r;
    v.resize(n);
    if (!r) {
        std::memcpy(v.data(), p, n * sizeof(double));
        return RSDFT_OK;
    }
    RS_CHECK(require_init());
    RS_CUDA(cudaMemcpyAsync(v.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, ctx().stream));
    RS_CUDA(cudaStreamSynchronize(ctx().stream));
    return RSDFT_OK;
}

// v into a host array or device memory at p.
int store_field(double* p, const std::vector<double>& v) {
    void* d = nullptr;
    const int r = resolve(p, v.size() * sizeof(double), &d);
    if (r < 0) return r;
    if (!r) {
        std::memcpy(p, v.data(), v.size() * sizeof(double));
        return RSDFT_OK;
    }
    RS_CHECK(require_init());
    RS_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, ctx().stream));
    RS_CUDA(cudaStreamSynchronize(ctx().stream));
    return RSDFT_OK;
}

}  // namespace
}  // namespace rsdft

extern "C" int rsdft_gpu_write_vrho(const char* path, const int* ngrid, const double* aa, int nelement, int natom,
                                    const double* aa_atom, const int* ki_atom, const int* zn_atom, double efermi,
                                    int nspin, const double* rho, const double* vloc, const double* vh,
                                    const double* vxc) {
    RS_ENTRY();
    if (!path || !ngrid || !aa || !rho || !vloc || !vh || !vxc || nspin < 1 || nelement < 0 || natom < 0 ||
        (natom > 0 && (!aa_atom || !ki_atom)) || (nelement > 0 && !zn_atom)) {
        set_error("write_vrho: NULL argument or bad counts");
        return RSDFT_EINVAL;
    }
    const int n1 = ngrid[0], n2 = ngrid[1], n3 = ngrid[2];
    if (n1 < 1 || n2 < 1 || n3 < 1) {
        set_error("write_vrho: bad grid %d x %d x %d", n1, n2, n3);
        return RSDFT_EINVAL;
    }
    const long ml = (long)n1 * n2 * n3;
    std::vector<double> f_rho, f_vloc, f_vh, f_vxc;
    RS_CHECK(fetch_field(rho, (size_t)ml * nspin, f_rho));
    RS_CHECK(fetch_field(vloc, (size_t)ml * nspin, f_vloc));
    RS_CHECK(fetch_field(vh, (size_t)ml, f_vh));
    RS_CHECK(fetch_field(vxc, (size_t)ml * nspin, f_vxc));

    File out;
    RS_CHECK(out.open(path, "wb"));
    RS_CHECK(write_values(out, text64("version3.0, comment_length=64")));
    RS_CHECK(write_values(out, std::vector<int32_t>{(int32_t)ml, n1, n2, n3}));
    std::vector<int32_t> ll2((size_t)3 * ml);
    for (long i = 0; i < ml; ++i) {
        ll2[3 * i] = (int32_t)(i % n1);
        ll2[3 * i + 1] = (int32_t)((i / n1) % n2);
        ll2[3 * i + 2] = (int32_t)(i / ((long)n1 * n2));
    }
    RS_CHECK(write_values(out, ll2));
    RS_CHECK(write_values(out, text64("lattice aa(3,3)")));
    RS_CHECK(write_values(out, std::vector<double>(aa, aa + 9)));
    RS_CHECK(write_values(out, text64("atom: Nelement Natom / aa_atom / ki_atom /zn_atom")));
    RS_CHECK(write_values(out, std::vector<int32_t>{nelement, natom}));
    RS_CHECK(write_record(out, {{aa_atom, sizeof(double) * 3 * (size_t)natom}}));
    RS_CHECK(write_record(out, {{ki_atom, sizeof(int32_t) * (size_t)natom}}));
    RS_CHECK(write_record(out, {{zn_atom, sizeof(int32_t) * (size_t)nelement}}));
    RS_CHECK(write_values(out, text64("Fermi energy")));
    RS_CHECK(write_values(out, std::vector<double>{efermi}));
    const size_t bytes = sizeof(double) * (size_t)ml;
    for (int s = 0; s < nspin; ++s) {
        const size_t o = (size_t)ml * s;
        RS_CHECK(write_record(out, {{f_rho.data() + o, bytes}}));
        RS_CHECK(write_record(out, {{f_vloc.data() + o, bytes}}));
        if (s == 0) RS_CHECK(write_record(out, {{f_vh.data(), bytes}}));
        RS_CHECK(write_record(out, {{f_vxc.data() + o, bytes}}));
    }
    return out.close();
}

extern "C" int rsdft_gpu_read_vrho(const char* path, const int* ngrid, int nspin, double* rho, double* vloc,
                                   double* vh, double* vxc, double* efermi) {
    RS_ENTRY();
    if (!path || !ngrid || nspin < 1) {
        set_error("read_vrho: NULL path/ngrid or bad nspin");
        return RSDFT_EINVAL;
    }
    const int n1 = ngrid[0], n2 = ngrid[1], n3 = ngrid[2];
    if (n1 < 1 || n2 < 1 || n3 < 1) {
        set_error("read_vrho: bad grid %d x %d x %d", n1, n2, n3);
        return RSDFT_EINVAL;
    }
    const long ml = (long)n1 * n2 * n3;
    File in;
    RS_CHECK(in.open(path, "rb"));
    // the version record, if any (read_data, io_module.f90:288-296)
    size_t len = 0;
    RS_CHECK(record_head(in, &len, "first"));
    const long body = ftell(in.f);
    char head[7] = {0};
    const bool versioned = len >= 7 && fread(head, 1, 7, in.f) == 7 && std::memcmp(head, "version", 7) == 0;
    if (fseek(in.f, versioned ? body + (long)len : body - 4, SEEK_SET) != 0) {
        set_error("'%s': seek failed in the first record", path);
        return RSDFT_EINVAL;
    }
    if (versioned) RS_CHECK(record_tail(in, len, "version"));
    int32_t dims[4];
    RS_CHECK(read_record(in, dims, sizeof(dims), "grid size"));
    if (dims[0] != ml || dims[1] != n1 || dims[2] != n2 || dims[3] != n3) {
        set_error("read_vrho: '%s' holds a %d x %d x %d grid (ML %d); the caller's is %d x %d x %d", path, dims[1],
                  dims[2], dims[3], dims[0], n1, n2, n3);
        return RSDFT_EINVAL;
    }
    std::vector<int32_t> ll2((size_t)3 * ml);
    RS_CHECK(read_record(in, ll2.data(), ll2.size() * sizeof(int32_t), "LL2"));
    std::vector<long> dst((size_t)ml);
    std::vector<char> seen((size_t)ml, 0);
    for (long i = 0; i < ml; ++i) {
        const int32_t i1 = ll2[3 * i], i2 = ll2[3 * i + 1], i3 = ll2[3 * i + 2];
        if (i1 < 0 || i1 >= n1 || i2 < 0 || i2 >= n2 || i3 < 0 || i3 >= n3) {
            set_error("read_vrho: '%s': LL2(:, %ld) = (%d, %d, %d) is off the grid", path, i + 1, i1, i2, i3);
            return RSDFT_EINVAL;
        }
        dst[i] = i1 + (long)n1 * (i2 + (long)n2 * i3);
        if (seen[dst[i]]++) {
            set_error("read_vrho: '%s': LL2 lists grid point (%d, %d, %d) twice", path, i1, i2, i3);
            return RSDFT_EINVAL;
        }
    }
    double ef = 0.0;
    if (versioned) {
        for (const char* w :
             {"lattice comment", "aa", "atom comment", "Nelement", "aa_atom", "ki_atom", "zn_atom", "Fermi comment"})
            RS_CHECK(skip_record(in, w));
        RS_CHECK(read_record(in, &ef, sizeof(ef), "efermi"));
    }
    std::vector<double> buf((size_t)ml), f_rho((size_t)ml * nspin), f_vloc((size_t)ml * nspin), f_vh((size_t)ml),
        f_vxc((size_t)ml * nspin);
    auto take = [&](std::vector<double>& f, size_t o, const char* what) -> int {
        RS_CHECK(read_record(in, buf.data(), sizeof(double) * (size_t)ml, what));
        for (long i = 0; i < ml; ++i) f[o + dst[i]] = buf[i];
        return RSDFT_OK;
    };
    for (int s = 0; s < nspin; ++s) {
        const size_t o = (size_t)ml * s;
        RS_CHECK(take(f_rho, o, "rho"));
        RS_CHECK(take(f_vloc, o, "Vloc"));
        if (s == 0) RS_CHECK(take(f_vh, 0, "Vh"));
        RS_CHECK(take(f_vxc, o, "Vxc"));
    }
    if (rho) RS_CHECK(store_field(rho, f_rho));
    if (vloc) RS_CHECK(store_field(vloc, f_vloc));
    if (vh) RS_CHECK(store_field(vh, f_vh));
    if (vxc) RS_CHECK(store_field(vxc, f_vxc));
    if (efermi && versioned) *efermi = ef;
    return RSDFT_OK;
}
