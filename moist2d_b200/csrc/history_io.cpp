// history_io.cpp - history and restart files of the large step's caller: init_history and
// output_history (moist.jl:1686-1891) and the restart read of run_sim (moist.jl:1905-1919).
//
// The reference writes through NCDatasets. This file writes the NetCDF classic format with
// 64-bit offsets (CDF-2, Unidata's published "NetCDF Classic and 64-bit Offset File Format")
// itself, so any NetCDF reader opens the result: a big-endian header (the dimensions x, z and
// the unlimited time; every variable with its "units" attribute), the fixed variables x, z, zf,
// then one record per output time holding every record variable in definition order. The
// variables, their order, dimensions and units are those of init_history; a Julia (x, z, time)
// variable is (time, z, x) in the file, x fastest, which is also the device layout.
//
// The restart reader parses the same format (CDF-1 or CDF-2 headers, attributes of any classic
// type, float or double variables) and fills a host State from the file's last record.
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/moist2d.h"

namespace {

thread_local std::string g_io_error;

int io_fail(const std::string& msg) {
    g_io_error = msg;
    return MOIST_ERR_IO;
}

enum { NC_BYTE = 1, NC_CHAR = 2, NC_SHORT = 3, NC_INT = 4, NC_FLOAT = 5, NC_DOUBLE = 6 };
enum { TAG_DIMENSION = 10, TAG_VARIABLE = 11, TAG_ATTRIBUTE = 12 };

// big-endian encoder
struct Enc {
    std::vector<unsigned char> b;
    void u32(uint32_t v) {
        for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void u64(uint64_t v) {
        for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void pad() {
        while (b.size() % 4) b.push_back(0);
    }
    void name(const std::string& s) {
        u32((uint32_t)s.size());
        b.insert(b.end(), s.begin(), s.end());
        pad();
    }
};

// element of type T (float or double) -> big-endian bytes
template <class T>
void put_be(unsigned char* dst, T v) {
    unsigned char raw[sizeof(T)];
    std::memcpy(raw, &v, sizeof(T));
    for (size_t j = 0; j < sizeof(T); j++) dst[j] = raw[sizeof(T) - 1 - j];
}

// The variables of init_history (moist.jl:1716-1788), in its order.
enum Kind { K_X, K_Z, K_TIME, K_XZ, K_X1 };  // x(x); z(z); time(time); (time, z, x); (time, x)
struct HVar {
    const char* name;
    Kind kind;
    const char* units;
};
const HVar HVARS[] = {
    {"x", K_X, "m"},
    {"z", K_Z, "m"},
    {"zf", K_Z, "m"},
    {"time", K_TIME, "s"},
    {"rho", K_XZ, "kg/m^3"},
    {"rhou", K_XZ, "kg/m^2/s"},
    {"rhow", K_XZ, "kg/m^2/s"},
    {"u", K_XZ, "m/s"},
    {"w", K_XZ, "m/s"},
    {"theta", K_XZ, "K"},
    {"qv", K_XZ, "kg/kg"},
    {"qc", K_XZ, "kg/kg"},
    {"qr", K_XZ, "kg/kg"},
    {"RH", K_XZ, "%"},
    {"temp", K_XZ, "K"},
    {"pres", K_XZ, "hPa"},
    {"thetae", K_XZ, "K"},
    {"prec", K_X1, "kg/m^2"},
    {"mflux", K_X1, "kg/m/s^2"},
    {"shflux", K_X1, "W/m^2"},
    {"lhflux", K_X1, "W/m^2"},
    {"d_rho_theta_mp", K_XZ, "kg K/m^3/s"},
    {"d_rho_qv_mp", K_XZ, "kg/m^3/s"},
    {"d_rho_qc_mp", K_XZ, "kg/m^3/s"},
    {"d_rho_qr_mp", K_XZ, "kg/m^3/s"},
    {"d_rho_qr_sed", K_XZ, "kg/m^3/s"},
    {"d_rho_u_sf", K_X1, "kg/m^2/s^2"},
    {"d_rho_theta_sf", K_X1, "kg K/m^3/s"},
    {"d_rho_qv_sf", K_X1, "kg/kg/m^3/s"},
    {"d_rho_theta_rd", K_XZ, "kg K/m^3/s"},
};
constexpr int NHVARS = (int)(sizeof(HVARS) / sizeof(HVARS[0]));

bool fseek64(FILE* f, uint64_t off) { return fseeko(f, (off_t)off, SEEK_SET) == 0; }

}  // namespace

struct moist_history {
    FILE* f = nullptr;
    std::string path;
    int prec = MOIST_F32;
    size_t es = 4;
    int nx = 0, nz = 0, halo = 0, ka = 0, ia = 0;
    uint32_t numrecs = 0;
    uint64_t recsize = 0;
    std::vector<uint64_t> begin;  // per HVARS entry
    std::vector<unsigned char> buf;
    // host staging of moist_history_append (allocated on first use)
    std::vector<std::vector<unsigned char>> st;
};

namespace {

uint64_t var_bytes(const moist_history* h, Kind k) {
    switch (k) {
        case K_X: return (uint64_t)h->nx * h->es;
        case K_Z: return (uint64_t)h->nz * h->es;
        case K_TIME: return h->es;
        case K_XZ: return (uint64_t)h->nx * h->nz * h->es;
        case K_X1: return (uint64_t)h->nx * h->es;
    }
    return 0;
}

// header with the given variable offsets (its length does not depend on them)
std::vector<unsigned char> header(const moist_history* h) {
    Enc e;
    e.b.insert(e.b.end(), {'C', 'D', 'F', 2});
    e.u32(h->numrecs);
    e.u32(TAG_DIMENSION);
    e.u32(3);
    e.name("x");
    e.u32((uint32_t)h->nx);
    e.name("z");
    e.u32((uint32_t)h->nz);
    e.name("time");
    e.u32(0);  // the record dimension
    e.u32(0);  // no global attributes
    e.u32(0);
    e.u32(TAG_VARIABLE);
    e.u32((uint32_t)NHVARS);
    for (int v = 0; v < NHVARS; v++) {
        const HVar& hv = HVARS[v];
        e.name(hv.name);
        switch (hv.kind) {
            case K_X: e.u32(1); e.u32(0); break;
            case K_Z: e.u32(1); e.u32(1); break;
            case K_TIME: e.u32(1); e.u32(2); break;
            case K_XZ: e.u32(3); e.u32(2); e.u32(1); e.u32(0); break;
            case K_X1: e.u32(2); e.u32(2); e.u32(0); break;
        }
        e.u32(TAG_ATTRIBUTE);
        e.u32(1);
        e.name("units");
        e.u32(NC_CHAR);
        e.name(hv.units);
        e.u32(h->prec == MOIST_F64 ? NC_DOUBLE : NC_FLOAT);
        e.u32((uint32_t)var_bytes(h, hv.kind));  // vsize (one record's worth for record variables)
        e.u64(h->begin.empty() ? 0 : h->begin[v]);
    }
    return e.b;
}

int write_at(moist_history* h, uint64_t off, const unsigned char* p, size_t n) {
    if (!fseek64(h->f, off) || fwrite(p, 1, n, h->f) != n)
        return io_fail(h->path + ": write failed: " + std::strerror(errno));
    return MOIST_OK;
}

// interior of a (ka, ia) column-major host field -> (z, x) rows, x fastest, big-endian
template <class T>
void pack_field(moist_history* h, const void* src) {
    const T* a = (const T*)src;
    h->buf.resize((size_t)h->nx * h->nz * sizeof(T));
    for (int k = 0; k < h->nz; k++)
        for (int i = 0; i < h->nx; i++)
            put_be(&h->buf[((size_t)k * h->nx + i) * sizeof(T)], a ? a[(size_t)(h->halo + i) * h->ka + k] : T(0));
}
// (Nz, Nx) z-fastest host array (moist_history_diagnostics) -> (z, x) rows
template <class T>
void pack_diag(moist_history* h, const void* src, bool to_hpa) {
    const T* a = (const T*)src;
    h->buf.resize((size_t)h->nx * h->nz * sizeof(T));
    for (int k = 0; k < h->nz; k++)
        for (int i = 0; i < h->nx; i++) {
            T v = a ? a[(size_t)i * h->nz + k] : T(0);
            if (to_hpa) v = v / T(100.0);  // Pa -> hPa, as output_history (moist.jl:1874)
            put_be(&h->buf[((size_t)k * h->nx + i) * sizeof(T)], v);
        }
}
// interior of an (ia) host vector
template <class T>
void pack_row(moist_history* h, const void* src) {
    const T* a = (const T*)src;
    h->buf.resize((size_t)h->nx * sizeof(T));
    for (int i = 0; i < h->nx; i++) put_be(&h->buf[(size_t)i * sizeof(T)], a ? a[h->halo + i] : T(0));
}

template <class T>
int create_t(moist_history* h, const moist_params* p) {
    // x: cell centres (i - is + 0.5) dx (moist.jl:203-205); z, zf: the grid vectors
    std::vector<unsigned char> xs((size_t)h->nx * sizeof(T)), zs((size_t)h->nz * sizeof(T)), zfs(zs.size());
    const T dx = (T)p->dx;
    for (int i = 0; i < h->nx; i++) put_be(&xs[(size_t)i * sizeof(T)], (T(i) + T(0.5)) * dx);
    for (int k = 0; k < h->nz; k++) {
        put_be(&zs[(size_t)k * sizeof(T)], ((const T*)p->z)[k]);
        put_be(&zfs[(size_t)k * sizeof(T)], ((const T*)p->zf)[k]);
    }
    const uint64_t hlen = header(h).size();
    h->begin.assign(NHVARS, 0);
    uint64_t off = hlen;
    for (int v = 0; v < NHVARS; v++)
        if (HVARS[v].kind == K_X || HVARS[v].kind == K_Z) {
            h->begin[v] = off;
            off += var_bytes(h, HVARS[v].kind);
        }
    h->recsize = 0;
    for (int v = 0; v < NHVARS; v++)
        if (!(HVARS[v].kind == K_X || HVARS[v].kind == K_Z)) {
            h->begin[v] = off + h->recsize;
            h->recsize += var_bytes(h, HVARS[v].kind);
        }
    const std::vector<unsigned char> hd = header(h);
    if (int r = write_at(h, 0, hd.data(), hd.size())) return r;
    if (int r = write_at(h, h->begin[0], xs.data(), xs.size())) return r;
    if (int r = write_at(h, h->begin[1], zs.data(), zs.size())) return r;
    if (int r = write_at(h, h->begin[2], zfs.data(), zfs.size())) return r;
    return fflush(h->f) == 0 ? MOIST_OK : io_fail(h->path + ": flush failed");
}

template <class T>
int append_t(moist_history* h, double t, const moist_state_host* s, const void* const diag[MOIST_NDIAG]) {
    const uint64_t r = h->numrecs;
    auto at = [&](int v) { return h->begin[v] + r * h->recsize; };
    for (int v = 0; v < NHVARS; v++) {
        const char* nm = HVARS[v].name;
        const Kind kd = HVARS[v].kind;
        if (kd == K_X || kd == K_Z) continue;
        if (kd == K_TIME) {
            h->buf.resize(sizeof(T));
            put_be(h->buf.data(), (T)t);
        } else if (!std::strcmp(nm, "rho")) {
            pack_field<T>(h, s->rho);
        } else if (!std::strcmp(nm, "rhou")) {
            pack_field<T>(h, s->rho_u);
        } else if (!std::strcmp(nm, "rhow")) {
            pack_field<T>(h, s->rho_w);
        } else if (!std::strcmp(nm, "u")) {
            pack_diag<T>(h, diag[MOIST_DIAG_U], false);
        } else if (!std::strcmp(nm, "w")) {
            pack_diag<T>(h, diag[MOIST_DIAG_W], false);
        } else if (!std::strcmp(nm, "theta")) {
            pack_diag<T>(h, diag[MOIST_DIAG_THETA], false);
        } else if (!std::strcmp(nm, "qv")) {
            pack_diag<T>(h, diag[MOIST_DIAG_QV], false);
        } else if (!std::strcmp(nm, "qc")) {
            pack_diag<T>(h, diag[MOIST_DIAG_QC], false);
        } else if (!std::strcmp(nm, "qr")) {
            pack_diag<T>(h, diag[MOIST_DIAG_QR], false);
        } else if (!std::strcmp(nm, "RH")) {
            pack_diag<T>(h, diag[MOIST_DIAG_RH], false);
        } else if (!std::strcmp(nm, "temp")) {
            pack_diag<T>(h, diag[MOIST_DIAG_TEMP], false);
        } else if (!std::strcmp(nm, "pres")) {
            pack_diag<T>(h, diag[MOIST_DIAG_PRES], true);
        } else if (!std::strcmp(nm, "thetae")) {
            pack_diag<T>(h, diag[MOIST_DIAG_THETAE], false);
        } else if (!std::strcmp(nm, "prec")) {
            pack_row<T>(h, s->prec);
        } else if (!std::strcmp(nm, "mflux")) {
            pack_row<T>(h, s->mflux);
        } else if (!std::strcmp(nm, "shflux")) {
            pack_row<T>(h, s->shflux);
        } else if (!std::strcmp(nm, "lhflux")) {
            pack_row<T>(h, s->lhflux);
        } else if (!std::strcmp(nm, "d_rho_theta_mp")) {
            pack_field<T>(h, s->d_rho_theta_mp);
        } else if (!std::strcmp(nm, "d_rho_qv_mp")) {
            pack_field<T>(h, s->d_rho_qv_mp);
        } else if (!std::strcmp(nm, "d_rho_qc_mp")) {
            pack_field<T>(h, s->d_rho_qc_mp);
        } else if (!std::strcmp(nm, "d_rho_qr_mp")) {
            pack_field<T>(h, s->d_rho_qr_mp);
        } else if (!std::strcmp(nm, "d_rho_qr_sed")) {
            // transposed like the other fields (the reference omits the transpose, moist.jl:1883)
            pack_field<T>(h, s->d_rho_qr_sed);
        } else if (!std::strcmp(nm, "d_rho_u_sf")) {
            pack_row<T>(h, s->d_rho_u_sf);
        } else if (!std::strcmp(nm, "d_rho_theta_sf")) {
            pack_row<T>(h, s->d_rho_theta_sf);
        } else if (!std::strcmp(nm, "d_rho_qv_sf")) {
            pack_row<T>(h, s->d_rho_qv_sf);
        } else if (!std::strcmp(nm, "d_rho_theta_rd")) {
            pack_field<T>(h, s->d_rho_theta_rd);
        }
        if (int rc = write_at(h, at(v), h->buf.data(), h->buf.size())) return rc;
    }
    // the record exists only once numrecs says so (sync(nc), moist.jl:1888)
    h->numrecs++;
    unsigned char nr[4];
    for (int j = 0; j < 4; j++) nr[j] = (unsigned char)(h->numrecs >> (24 - 8 * j));
    if (int rc = write_at(h, 4, nr, 4)) return rc;
    return fflush(h->f) == 0 ? MOIST_OK : io_fail(h->path + ": flush failed");
}

// ------------------------------------------------------------------------------- reader

struct NcVar {
    std::string name;
    std::vector<uint32_t> dims;
    uint32_t type = 0;
    uint64_t vsize = 0, begin = 0;
};
struct NcFile {
    FILE* f = nullptr;
    std::string path;
    int version = 0;
    uint32_t numrecs = 0;
    std::vector<std::pair<std::string, uint32_t>> dims;
    std::vector<NcVar> vars;
    uint64_t recsize = 0;
    ~NcFile() {
        if (f) fclose(f);
    }
    bool u32(uint32_t* v) {
        unsigned char b[4];
        if (fread(b, 1, 4, f) != 4) return false;
        *v = ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
        return true;
    }
    bool u64(uint64_t* v) {
        uint32_t hi, lo;
        if (!u32(&hi) || !u32(&lo)) return false;
        *v = ((uint64_t)hi << 32) | lo;
        return true;
    }
    bool skip(uint64_t n) { return fseeko(f, (off_t)n, SEEK_CUR) == 0; }
    bool name(std::string* s) {
        uint32_t n;
        if (!u32(&n) || n > (1u << 20)) return false;
        s->resize(n);
        if (n && fread(&(*s)[0], 1, n, f) != n) return false;
        return skip((4 - n % 4) % 4);
    }
    static uint64_t type_size(uint32_t t) {
        switch (t) {
            case NC_BYTE: case NC_CHAR: return 1;
            case NC_SHORT: return 2;
            case NC_INT: case NC_FLOAT: return 4;
            case NC_DOUBLE: return 8;
        }
        return 0;
    }
    bool skip_atts() {
        uint32_t tag, n;
        if (!u32(&tag) || !u32(&n)) return false;
        if (tag == 0 && n == 0) return true;
        if (tag != TAG_ATTRIBUTE) return false;
        for (uint32_t a = 0; a < n; a++) {
            std::string nm;
            uint32_t t, ne;
            if (!name(&nm) || !u32(&t) || !u32(&ne)) return false;
            const uint64_t sz = type_size(t);
            if (!sz) return false;
            const uint64_t bytes = sz * ne;
            if (!skip(bytes + (4 - bytes % 4) % 4)) return false;
        }
        return true;
    }
    int open(const char* p) {
        path = p;
        f = fopen(p, "rb");
        if (!f) return io_fail(path + ": cannot open: " + std::strerror(errno));
        unsigned char magic[4];
        if (fread(magic, 1, 4, f) != 4 || magic[0] != 'C' || magic[1] != 'D' || magic[2] != 'F' ||
            (magic[3] != 1 && magic[3] != 2))
            return io_fail(path + ": not a NetCDF classic or 64-bit offset file");
        version = magic[3];
        if (!u32(&numrecs)) return io_fail(path + ": truncated header");
        if (numrecs == 0xFFFFFFFFu) return io_fail(path + ": record count not finalised (streaming)");
        uint32_t tag, n;
        if (!u32(&tag) || !u32(&n)) return io_fail(path + ": truncated header");
        if (tag == TAG_DIMENSION) {
            for (uint32_t d = 0; d < n; d++) {
                std::string nm;
                uint32_t len;
                if (!name(&nm) || !u32(&len)) return io_fail(path + ": bad dimension list");
                dims.push_back({nm, len});
            }
        } else if (tag != 0 || n != 0) {
            return io_fail(path + ": bad dimension list");
        }
        if (!skip_atts()) return io_fail(path + ": bad global attribute list");
        if (!u32(&tag) || !u32(&n)) return io_fail(path + ": truncated header");
        if (tag == TAG_VARIABLE) {
            for (uint32_t v = 0; v < n; v++) {
                NcVar var;
                uint32_t nd, vs;
                if (!name(&var.name) || !u32(&nd) || nd > 64) return io_fail(path + ": bad variable list");
                var.dims.resize(nd);
                for (uint32_t d = 0; d < nd; d++)
                    if (!u32(&var.dims[d]) || var.dims[d] >= dims.size()) return io_fail(path + ": bad variable list");
                if (!skip_atts() || !u32(&var.type) || !u32(&vs)) return io_fail(path + ": bad variable list");
                var.vsize = vs;
                if (version == 1) {
                    uint32_t b;
                    if (!u32(&b)) return io_fail(path + ": bad variable list");
                    var.begin = b;
                } else if (!u64(&var.begin)) {
                    return io_fail(path + ": bad variable list");
                }
                vars.push_back(var);
            }
        } else if (tag != 0 || n != 0) {
            return io_fail(path + ": bad variable list");
        }
        // record size: the record variables' vsizes; a lone record variable is not padded
        int nrec = 0;
        uint64_t lone = 0;
        for (const NcVar& v : vars)
            if (is_record(v)) {
                nrec++;
                recsize += v.vsize;
                lone = 1;
                for (size_t d = 1; d < v.dims.size(); d++) lone *= dims[v.dims[d]].second;
                lone *= type_size(v.type);
            }
        if (nrec == 1) recsize = lone;
        return MOIST_OK;
    }
    bool is_record(const NcVar& v) const { return !v.dims.empty() && dims[v.dims[0]].second == 0; }
    const NcVar* find(const char* nm) const {
        for (const NcVar& v : vars)
            if (v.name == nm) return &v;
        return nullptr;
    }
    // record r of a record variable whose other dimensions have the given lengths, as doubles
    // (float values widen exactly); *is_double tells the stored type
    int read_record(const char* nm, uint32_t r, const std::vector<uint32_t>& shape, std::vector<double>* out,
                    bool* is_double) {
        const NcVar* v = find(nm);
        if (!v) return io_fail(path + ": no variable \"" + nm + "\"");
        if (!is_record(*v) || v->dims.size() != shape.size() + 1)
            return io_fail(path + ": variable \"" + nm + "\" has other dimensions than expected");
        uint64_t n = 1;
        for (size_t d = 0; d < shape.size(); d++) {
            if (dims[v->dims[d + 1]].second != shape[d])
                return io_fail(path + ": variable \"" + nm + "\" has other dimension lengths than the Params");
            n *= shape[d];
        }
        if (v->type != NC_FLOAT && v->type != NC_DOUBLE)
            return io_fail(path + ": variable \"" + nm + "\" is neither float nor double");
        *is_double = v->type == NC_DOUBLE;
        const uint64_t es = *is_double ? 8 : 4;
        std::vector<unsigned char> raw(n * es);
        if (fseeko(f, (off_t)(v->begin + (uint64_t)r * recsize), SEEK_SET) != 0 ||
            fread(raw.data(), 1, raw.size(), f) != raw.size())
            return io_fail(path + ": variable \"" + nm + "\" is truncated");
        out->resize(n);
        for (uint64_t j = 0; j < n; j++) {
            unsigned char b[8];
            for (uint64_t q = 0; q < es; q++) b[q] = raw[j * es + es - 1 - q];
            if (*is_double) {
                double d;
                std::memcpy(&d, b, 8);
                (*out)[j] = d;
            } else {
                float x;
                std::memcpy(&x, b, 4);
                (*out)[j] = x;
            }
        }
        return MOIST_OK;
    }
};

// a * b in the file's type F, rounded to the State's type T: the arithmetic of
// state.rho_theta[...] = nc["theta"][...]' .* rho (moist.jl:1914-1917)
template <class T>
T prod_in(bool file_double, double a, double b) {
    return file_double ? (T)(a * b) : (T)((float)a * (float)b);
}

template <class T>
int restart_t(NcFile& nc, const moist_params* p, moist_state_host* s) {
    const int nx = p->nx, nz = p->nz, halo = p->halo, ka = nz, ia = nx + 2 * halo;
    if (nc.numrecs == 0) return io_fail(nc.path + ": the file holds no record");
    const uint32_t r = nc.numrecs - 1;
    const std::vector<uint32_t> zx = {(uint32_t)nz, (uint32_t)nx}, x1 = {(uint32_t)nx};
    std::vector<double> rho, f;
    bool drho, df;
    if (int rc = nc.read_record("rho", r, zx, &rho, &drho)) return rc;
    auto put = [&](void* dst, auto value_of) {
        T* a = (T*)dst;
        for (int k = 0; k < nz; k++)
            for (int i = 0; i < nx; i++) a[(size_t)(halo + i) * ka + k] = value_of((size_t)k * nx + i);
        // exchange_halo! (moist.jl:233-241), as run_sim does after the restart (1927-1929):
        // both source strips are read before either halo is written
        std::vector<T> left((size_t)ka * halo), right((size_t)ka * halo);
        for (int hh = 0; hh < halo; hh++)
            for (int k = 0; k < ka; k++) {
                left[(size_t)hh * ka + k] = a[(size_t)(nx + hh) * ka + k];
                right[(size_t)hh * ka + k] = a[(size_t)(halo + hh) * ka + k];
            }
        for (int hh = 0; hh < halo; hh++)
            for (int k = 0; k < ka; k++) {
                a[(size_t)hh * ka + k] = left[(size_t)hh * ka + k];
                a[(size_t)(halo + nx + hh) * ka + k] = right[(size_t)hh * ka + k];
            }
    };
    if (s->rho) put(s->rho, [&](size_t j) { return (T)rho[j]; });
    struct Plain { const char* nm; void* dst; };
    const Plain plain[] = {{"rhou", s->rho_u}, {"rhow", s->rho_w}};
    for (const Plain& q : plain) {
        if (!q.dst) continue;
        if (int rc = nc.read_record(q.nm, r, zx, &f, &df)) return rc;
        put(q.dst, [&](size_t j) { return (T)f[j]; });
    }
    // mixing ratios times rho; rho_qr from "qr" (the reference reads "qc" there, moist.jl:1917)
    const Plain mixed[] = {{"theta", s->rho_theta}, {"qv", s->rho_qv}, {"qc", s->rho_qc}, {"qr", s->rho_qr}};
    for (const Plain& q : mixed) {
        if (!q.dst) continue;
        if (int rc = nc.read_record(q.nm, r, zx, &f, &df)) return rc;
        if (df != drho) return io_fail(nc.path + ": \"" + q.nm + "\" and \"rho\" differ in type");
        put(q.dst, [&](size_t j) { return prod_in<T>(drho, f[j], rho[j]); });
    }
    if (s->prec) {
        if (int rc = nc.read_record("prec", r, x1, &f, &df)) return rc;
        T* a = (T*)s->prec;
        for (int i = 0; i < nx; i++) a[halo + i] = (T)f[i];
    }
    return MOIST_OK;
}

}  // namespace

extern "C" {
#pragma GCC visibility push(default)

const char* moist_io_last_error(void) { return g_io_error.c_str(); }

int moist_history_create(const char* path, const moist_params* p, int precision, moist_history** out) {
    if (!out) return MOIST_ERR_ARG;
    *out = nullptr;
    if (!path || !p || !p->z || !p->zf || p->nx < 1 || p->nz < 1 || p->halo < 0 ||
        (precision != MOIST_F32 && precision != MOIST_F64))
        return MOIST_ERR_ARG;
    // a CDF-2 variable's per-record size is a 32-bit field
    if ((uint64_t)p->nx * (uint64_t)p->nz * (precision == MOIST_F64 ? 8u : 4u) >= 0xFFFFFFFCull) return MOIST_ERR_ARG;
    moist_history* h = new moist_history;
    h->path = path;
    h->prec = precision;
    h->es = precision == MOIST_F64 ? 8 : 4;
    h->nx = p->nx;
    h->nz = p->nz;
    h->halo = p->halo;
    h->ka = p->nz;
    h->ia = p->nx + 2 * p->halo;
    // an existing file is replaced (moist.jl:1718)
    h->f = fopen(path, "w+b");
    if (!h->f) {
        const int rc = io_fail(std::string(path) + ": cannot create: " + std::strerror(errno));
        delete h;
        return rc;
    }
    const int rc = precision == MOIST_F64 ? create_t<double>(h, p) : create_t<float>(h, p);
    if (rc) {
        fclose(h->f);
        delete h;
        return rc;
    }
    *out = h;
    return MOIST_OK;
}

int moist_history_append_host(moist_history* h, double t, const moist_state_host* s,
                              const void* const diag[MOIST_NDIAG]) {
    if (!h || !s || !diag) return MOIST_ERR_ARG;
    return h->prec == MOIST_F64 ? append_t<double>(h, t, s, diag) : append_t<float>(h, t, s, diag);
}

int moist_history_append(moist_history* h, double t, moist_ctx* ctx) {
    if (!h || !ctx) return MOIST_ERR_ARG;
    const size_t es = h->es, f2 = (size_t)h->ka * h->ia * es, f1 = (size_t)h->ia * es, fk = (size_t)h->ka * es;
    const size_t sizes[21] = {f2, f2, f2, f2, f2, f2, f2, f1, f1, f1, f1, fk, f2, f2, f2, f2, f2, f1, f1, f1, f2};
    if (h->st.empty()) {
        h->st.resize(21 + MOIST_NDIAG);
        for (int j = 0; j < 21; j++) h->st[j].assign(sizes[j], 0);
        for (int j = 0; j < MOIST_NDIAG; j++) h->st[21 + j].assign((size_t)h->nx * h->nz * es, 0);
    }
    void* b[21];
    for (int j = 0; j < 21; j++) b[j] = h->st[j].data();
    moist_state_host s = {b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8], b[9], b[10],
                          b[11], b[12], b[13], b[14], b[15], b[16], b[17], b[18], b[19], b[20]};
    if (int rc = moist_download_state(ctx, &s)) return rc;
    void* d[MOIST_NDIAG];
    for (int j = 0; j < MOIST_NDIAG; j++) d[j] = h->st[21 + j].data();
    if (int rc = moist_history_diagnostics(ctx, d, nullptr)) return rc;
    return moist_history_append_host(h, t, &s, d);
}

int moist_history_close(moist_history* h) {
    if (!h) return MOIST_OK;
    const int rc = fclose(h->f) == 0 ? MOIST_OK : io_fail(h->path + ": close failed");
    delete h;
    return rc;
}

int moist_restart_read(const char* path, const moist_params* p, int precision, moist_state_host* s) {
    if (!path || !p || !s || p->nx < 1 || p->nz < 1 || p->halo < 0 ||
        (precision != MOIST_F32 && precision != MOIST_F64))
        return MOIST_ERR_ARG;
    NcFile nc;
    if (int rc = nc.open(path)) return rc;
    return precision == MOIST_F64 ? restart_t<double>(nc, p, s) : restart_t<float>(nc, p, s);
}

#pragma GCC visibility pop
}  // extern "C"
