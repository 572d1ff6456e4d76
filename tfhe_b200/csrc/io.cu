// io.cu -- gate-bootstrapping parameter sets, key sets and ciphertexts in the reference's file
// format (tfhe_io.cpp, tfhe_generic_streams.cpp), so that keys and ciphertexts written by an
// existing tfhe installation load here and the other way round.
//
// A file is a sequence of text sections and binary blocks, in this order:
//   parameter set  GATEBOOTSPARAMS, LWEPARAMS, TLWEPARAMS, TGSWPARAMS        (tfhe_io.cpp:1010-1041)
//   cloud key set  parameter set, LWEKSPARAMS, keyswitch block, bootstrapping block (:1103-1122)
//   secret key set cloud key set, LWE key block, TGSW key block           (:1157-1176)
//   ciphertext     LWE sample block                                       (:90-110, :1211-1220)
// Text section (tfhe_generic_streams.cpp:119-176): "-----BEGIN T-----", one "name: value" line per
// property in ascending name order, "-----END T-----"; integers as "%10" PRId64, reals as "%.8lf".
// Binary blocks (native byte order): an int32 type id, then
//   keyswitch (200):     double max variance, then [kN][t][base] samples of n+1 int32 (a, b)
//   bootstrapping (201): double max variance, then [n][(k+1)l][k+1] polynomials of N int32
//   LWE key (43):        n int32;   TGSW key (169): k polynomials of N int32
//   LWE sample (42):     n int32 (a), int32 (b), double (variance)
// These are exactly the engine's raw key layouts, so loading is a copy.
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "internal.h"

namespace tfheb {
namespace io {

namespace {

constexpr int32_t kLweSampleUid = 42, kLweKeyUid = 43, kTgswKeyUid = 169, kKeySwitchUid = 200,
                  kBootstrapUid = 201;  // tfhe_generic_streams.h:15-30

struct Section {
    std::string title;
    std::map<std::string, std::string> kv;  // ordered by name, as the reference prints them
};

std::string fmt_int(int64_t v) {
    char b[64];
    std::snprintf(b, sizeof b, "%10" PRId64, v);
    return b;
}
std::string fmt_real(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.8lf", v);
    return b;
}

bool write_section(FILE *f, const Section &s) {
    std::string out = "-----BEGIN " + s.title + "-----\n";
    for (const auto &it : s.kv) out += it.first + ": " + it.second + "\n";
    out += "-----END " + s.title + "-----\n";
    return std::fwrite(out.data(), 1, out.size(), f) == out.size();
}

// one line without its '\n'; '\r' dropped; false at end of file with nothing read
bool read_line(FILE *f, std::string &line) {
    line.clear();
    bool any = false;
    for (int c = std::fgetc(f); c != EOF; c = std::fgetc(f)) {
        any = true;
        if (c == '\r') continue;
        if (c == '\n') return true;
        line.push_back((char)c);
    }
    return any;
}

// Next section; lines before "-----BEGIN" and lines without ": " are skipped, as in the reference.
bool read_section(FILE *f, Section &s) {
    std::string line, end;
    bool started = false;
    s.kv.clear();
    while (read_line(f, line)) {
        const size_t n = line.size();
        if (n >= 16 && line.compare(0, 11, "-----BEGIN ") == 0 && line.compare(n - 5, 5, "-----") == 0) {
            s.title = line.substr(11, n - 16);
            end = "-----END " + s.title + "-----";
            started = true;
            continue;
        }
        if (!started) continue;
        if (line == end) return true;
        const size_t pos = line.find(": ");
        if (pos == std::string::npos) continue;
        s.kv[line.substr(0, pos)] = line.substr(pos + 2);
    }
    return false;
}

bool get_int(const Section &s, const char *name, int64_t &v) {
    auto it = s.kv.find(name);
    if (it == s.kv.end()) return false;
    char *e = nullptr;
    v = std::strtoll(it->second.c_str(), &e, 10);
    return e != it->second.c_str();
}
bool get_real(const Section &s, const char *name, double &v) {
    auto it = s.kv.find(name);
    if (it == s.kv.end()) return false;
    char *e = nullptr;
    v = (double)std::strtold(it->second.c_str(), &e);
    return e != it->second.c_str();
}

template <typename T>
bool put(FILE *f, const T *v, size_t count) {
    return std::fwrite(v, sizeof(T), count, f) == count;
}
template <typename T>
bool get(FILE *f, T *v, size_t count) {
    return std::fread(v, sizeof(T), count, f) == count;
}
bool expect_uid(FILE *f, int32_t uid, const char *what) {
    int32_t got = 0;
    if (!get(f, &got, 1) || got != uid) {
        set_error(std::string("not a ") + what + " block (type id " + std::to_string(got) + ", expected " +
                  std::to_string(uid) + ")");
        return false;
    }
    return true;
}
bool fail(const std::string &msg) {
    set_error(msg);
    return false;
}

}  // namespace

// ---- parameter set (tfhe_io.cpp:35-60, 243-270, 480-520, 1010-1041) --------------------------

bool write_params(FILE *f, const tfheb_params &p, const ParamMeta &m) {
    Section g{"GATEBOOTSPARAMS", {{"ks_t", fmt_int(p.ks_t)}, {"ks_basebit", fmt_int(p.ks_basebit)}}};
    Section l{"LWEPARAMS",
              {{"n", fmt_int(p.n)}, {"alpha_min", fmt_real(p.ks_stdev)}, {"alpha_max", fmt_real(m.in_alpha_max)}}};
    Section t{"TLWEPARAMS",
              {{"N", fmt_int(p.N)},
               {"k", fmt_int(p.k)},
               {"alpha_min", fmt_real(p.bk_stdev)},
               {"alpha_max", fmt_real(m.tlwe_alpha_max)}}};
    Section w{"TGSWPARAMS", {{"l", fmt_int(p.l)}, {"Bgbit", fmt_int(p.Bgbit)}}};
    return write_section(f, g) && write_section(f, l) && write_section(f, t) && write_section(f, w);
}

bool read_params(FILE *f, tfheb_params &p, ParamMeta &m) {
    Section s;
    int64_t v;
    double d;
    if (!read_section(f, s) || s.title != "GATEBOOTSPARAMS") return fail("expected a GATEBOOTSPARAMS section");
    if (!get_int(s, "ks_t", v)) return fail("GATEBOOTSPARAMS without ks_t");
    p.ks_t = (int32_t)v;
    // the reference reads ks_basebit as a real (tfhe_io.cpp:1019)
    if (!get_real(s, "ks_basebit", d)) return fail("GATEBOOTSPARAMS without ks_basebit");
    p.ks_basebit = (int32_t)d;
    if (!read_section(f, s) || s.title != "LWEPARAMS") return fail("expected a LWEPARAMS section");
    if (!get_int(s, "n", v) || !get_real(s, "alpha_min", p.ks_stdev) || !get_real(s, "alpha_max", m.in_alpha_max))
        return fail("incomplete LWEPARAMS section");
    p.n = (int32_t)v;
    if (!read_section(f, s) || s.title != "TLWEPARAMS") return fail("expected a TLWEPARAMS section");
    if (!get_int(s, "N", v)) return fail("TLWEPARAMS without N");
    p.N = (int32_t)v;
    if (!get_int(s, "k", v) || !get_real(s, "alpha_min", p.bk_stdev) || !get_real(s, "alpha_max", m.tlwe_alpha_max))
        return fail("incomplete TLWEPARAMS section");
    p.k = (int32_t)v;
    if (!read_section(f, s) || s.title != "TGSWPARAMS") return fail("expected a TGSWPARAMS section");
    if (!get_int(s, "l", v)) return fail("TGSWPARAMS without l");
    p.l = (int32_t)v;
    if (!get_int(s, "Bgbit", v)) return fail("TGSWPARAMS without Bgbit");
    p.Bgbit = (int32_t)v;
    return true;
}

// ---- cloud key set content: keyswitch and bootstrapping keys (tfhe_io.cpp:731-817, 883-975) ---

bool write_cloud_content(FILE *f, const CloudKey &ck) {
    const tfheb_params &p = ck.p;
    if (ck.ksk.empty()) return fail("the cloud key has no keyswitching key to save");
    Section s{"LWEKSPARAMS",
              {{"n", fmt_int((int64_t)p.k * p.N)}, {"t", fmt_int(p.ks_t)}, {"basebit", fmt_int(p.ks_basebit)}}};
    const double ks_var = ck.ks_var >= 0 ? ck.ks_var : p.ks_stdev * p.ks_stdev;
    const double bk_var = ck.bk_var >= 0 ? ck.bk_var : p.bk_stdev * p.bk_stdev;
    return write_section(f, s) && put(f, &kKeySwitchUid, 1) && put(f, &ks_var, 1) &&
           put(f, ck.ksk.data(), ck.ksk.size()) && put(f, &kBootstrapUid, 1) && put(f, &bk_var, 1) &&
           put(f, ck.bsk_coef.data(), ck.bsk_coef.size());
}

// p: the parameter set read before; its keyswitch length and base come from the key's own section
bool read_cloud_content(FILE *f, tfheb_params &p, CloudKey &ck) {
    Section s;
    int64_t n, t, basebit;
    if (!read_section(f, s) || s.title != "LWEKSPARAMS") return fail("expected a LWEKSPARAMS section");
    if (!get_int(s, "n", n) || !get_int(s, "t", t) || !get_int(s, "basebit", basebit))
        return fail("incomplete LWEKSPARAMS section");
    if (n != (int64_t)p.k * p.N) return fail("Wrong dimension in bootstrapping key");  // tfhe_io.cpp:961
    if (t <= 0 || basebit <= 0 || t * basebit > 31) return fail("invalid keyswitch parameters");
    p.ks_t = (int32_t)t;
    p.ks_basebit = (int32_t)basebit;
    ck.p = p;
    ck.ksk.resize((size_t)n * t * ((size_t)1 << basebit) * (p.n + 1));
    ck.bsk_coef.resize((size_t)p.n * (p.k + 1) * p.l * (p.k + 1) * p.N);
    if (!expect_uid(f, kKeySwitchUid, "keyswitching key")) return false;
    if (!get(f, &ck.ks_var, 1) || !get(f, ck.ksk.data(), ck.ksk.size())) return fail("truncated keyswitching key");
    if (!expect_uid(f, kBootstrapUid, "bootstrapping key")) return false;
    if (!get(f, &ck.bk_var, 1) || !get(f, ck.bsk_coef.data(), ck.bsk_coef.size()))
        return fail("truncated bootstrapping key");
    return true;
}

// ---- secret key content: LWE key, then TGSW key (tfhe_io.cpp:154-205, 644-693) ---------------

bool write_secret_content(FILE *f, const SecretKey &sk) {
    return put(f, &kLweKeyUid, 1) && put(f, sk.lwe_key.data(), sk.lwe_key.size()) && put(f, &kTgswKeyUid, 1) &&
           put(f, sk.tlwe_key.data(), sk.tlwe_key.size());
}

bool read_secret_content(FILE *f, const tfheb_params &p, SecretKey &sk) {
    sk.p = p;
    sk.lwe_key.resize(p.n);
    sk.tlwe_key.resize((size_t)p.k * p.N);
    if (!expect_uid(f, kLweKeyUid, "LWE key")) return false;
    if (!get(f, sk.lwe_key.data(), sk.lwe_key.size())) return fail("truncated LWE key");
    if (!expect_uid(f, kTgswKeyUid, "TGSW key")) return false;
    if (!get(f, sk.tlwe_key.data(), sk.tlwe_key.size())) return fail("truncated TGSW key");
    return true;
}

// ---- LWE samples (tfhe_io.cpp:90-110) ---------------------------------------------------------

bool write_lwe_sample(FILE *f, int32_t n, const int32_t *a, int32_t b, double variance) {
    return put(f, &kLweSampleUid, 1) && put(f, a, (size_t)n) && put(f, &b, 1) && put(f, &variance, 1);
}

bool read_lwe_sample(FILE *f, int32_t n, int32_t *a, int32_t *b, double *variance) {
    if (!expect_uid(f, kLweSampleUid, "LWE sample")) return false;
    double v = 0;
    if (!get(f, a, (size_t)n) || !get(f, b, 1) || !get(f, &v, 1)) return fail("truncated LWE sample");
    if (variance) *variance = v;
    return true;
}

}  // namespace io
}  // namespace tfheb

// ================================================================================================
// native C ABI: path-based forms of the same files
// ================================================================================================

using namespace tfheb;

namespace {

struct File {
    FILE *f;
    File(const char *path, const char *mode) : f(path ? std::fopen(path, mode) : nullptr) {}
    ~File() {
        if (f) std::fclose(f);
    }
    bool close() {  // flushes; false when the data did not reach the file
        const bool ok = std::fclose(f) == 0;
        f = nullptr;
        return ok;
    }
};

tfheb_status open_error(const char *path) {
    set_error(std::string("cannot open ") + (path ? path : "(null)"));
    return TFHEB_ERR_INVALID;
}

bool params_ok(const tfheb_params &p) {
    return p.n > 0 && p.N > 0 && (p.N & (p.N - 1)) == 0 && p.k > 0 && p.l > 0 && p.Bgbit > 0 &&
           p.l * p.Bgbit <= 32 && p.ks_t > 0 && p.ks_basebit > 0 && p.ks_t * p.ks_basebit <= 31;
}

}  // namespace

extern "C" {

tfheb_status tfheb_params_save(const char *path, const tfheb_params *p) {
    if (!p) return TFHEB_ERR_INVALID;
    File F(path, "wb");
    if (!F.f) return open_error(path);
    if (!io::write_params(F.f, *p, ParamMeta{}) || !F.close()) return TFHEB_ERR_INVALID;
    return TFHEB_OK;
}

tfheb_status tfheb_params_load(const char *path, tfheb_params *p) {
    if (!p) return TFHEB_ERR_INVALID;
    File F(path, "rb");
    if (!F.f) return open_error(path);
    tfheb_params q{};
    ParamMeta m;
    if (!io::read_params(F.f, q, m)) return TFHEB_ERR_INVALID;
    if (!params_ok(q)) {
        set_error("parameter set out of range");
        return TFHEB_ERR_INVALID;
    }
    *p = q;
    return TFHEB_OK;
}

tfheb_status tfheb_cloud_key_save(const tfheb_cloud_key *ck, const char *path) {
    if (!ck) return TFHEB_ERR_INVALID;
    File F(path, "wb");
    if (!F.f) return open_error(path);
    if (!io::write_params(F.f, ck->ck.p, ck->ck.meta) || !io::write_cloud_content(F.f, ck->ck) || !F.close())
        return TFHEB_ERR_INVALID;
    return TFHEB_OK;
}

tfheb_status tfheb_cloud_key_load(const char *path, tfheb_cloud_key **out) {
    if (!out) return TFHEB_ERR_INVALID;
    File F(path, "rb");
    if (!F.f) return open_error(path);
    tfheb_params p{};
    auto *c = new tfheb_cloud_key();
    if (!io::read_params(F.f, p, c->ck.meta) || !params_ok(p) || !io::read_cloud_content(F.f, p, c->ck)) {
        delete c;
        return TFHEB_ERR_INVALID;
    }
    *out = c;
    return TFHEB_OK;
}

tfheb_status tfheb_secret_keyset_save(const tfheb_secret_key *sk, const tfheb_cloud_key *ck, const char *path) {
    if (!sk || !ck) return TFHEB_ERR_INVALID;
    File F(path, "wb");
    if (!F.f) return open_error(path);
    if (!io::write_params(F.f, ck->ck.p, ck->ck.meta) || !io::write_cloud_content(F.f, ck->ck) ||
        !io::write_secret_content(F.f, sk->sk) || !F.close())
        return TFHEB_ERR_INVALID;
    return TFHEB_OK;
}

tfheb_status tfheb_secret_keyset_load(const char *path, tfheb_secret_key **sk, tfheb_cloud_key **ck) {
    if (!sk || !ck) return TFHEB_ERR_INVALID;
    File F(path, "rb");
    if (!F.f) return open_error(path);
    tfheb_params p{};
    auto *c = new tfheb_cloud_key();
    auto *s = new tfheb_secret_key();
    if (!io::read_params(F.f, p, c->ck.meta) || !params_ok(p) || !io::read_cloud_content(F.f, p, c->ck) ||
        !io::read_secret_content(F.f, p, s->sk)) {
        delete c;
        delete s;
        return TFHEB_ERR_INVALID;
    }
    *sk = s;
    *ck = c;
    return TFHEB_OK;
}

tfheb_status tfheb_ciphertexts_save(const char *path, const tfheb_params *p, int32_t count, const int32_t *cts,
                                    const double *variances) {
    if (!p || count < 0 || (count > 0 && !cts)) return TFHEB_ERR_INVALID;
    File F(path, "wb");
    if (!F.f) return open_error(path);
    for (int32_t g = 0; g < count; g++) {
        const int32_t *c = cts + (size_t)g * (p->n + 1);
        if (!io::write_lwe_sample(F.f, p->n, c, c[p->n], variances ? variances[g] : 0.0)) return TFHEB_ERR_INVALID;
    }
    return F.close() ? TFHEB_OK : TFHEB_ERR_INVALID;
}

tfheb_status tfheb_ciphertexts_load(const char *path, const tfheb_params *p, int32_t count, int32_t *cts,
                                    double *variances) {
    if (!p || count < 0 || (count > 0 && !cts)) return TFHEB_ERR_INVALID;
    File F(path, "rb");
    if (!F.f) return open_error(path);
    for (int32_t g = 0; g < count; g++) {
        int32_t *c = cts + (size_t)g * (p->n + 1);
        if (!io::read_lwe_sample(F.f, p->n, c, c + p->n, variances ? variances + g : nullptr))
            return TFHEB_ERR_INVALID;
    }
    return TFHEB_OK;
}

}  // extern "C"
