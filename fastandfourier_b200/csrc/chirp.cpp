// chirp.cpp -- the Chirp forms of the transform path: S-expression reader,
// spectral-callback registry, chirp_bind, and chirp_compile for (fft),
// (ifft), (rfft), (irfft) and the fused (pipeline (rfft ..) OPS .. (irfft)).
//
// Grammar and defaults follow the reference compiler (src/chirp.c:529-890
// lexer/parser, :1642-1727 rfft/fft nodes, :1853-2055 pipeline, :2058-2135
// dispatch): keywords are `:name value` or bare flags (`:bluestein`);
// (fft) defaults to INTERLEAVED layout; (rfft) to HERMITIAN; size defaults
// to 64; a pipeline's middle forms must be spectral ops; the inverse half
// is (irfft [...]) or (inverse).  The emitted transform has the reference's
// shape: type PIPELINE, inner = forward R2C, inner_inv = C2R, code[i] =
// CALL_BUILTIN with a0 = CHIRP_OP_* or a registry index.
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "chirp.h"
#include "faf_api_internal.h"
#include "faf_cuda.h"

using namespace fafapi;

namespace {

// ---- registry (reference src/chirp.c:314-386) ----------------------------

struct Builtin {
    std::string name;
    chirp_spectral_fn f32 = nullptr;
    chirp_spectral_fn_f64 f64 = nullptr;
    int kind = CHIRP_KIND_SPECTRAL;
    void* ctx = nullptr;
    bool device = false;  // chirp_register_spectral_device: runs in the fused kernel
    int dop = 0;          // chirp_device_op
    double p0 = 0;
};

// Phase of the circular delay at bin k of an n-point transform: -2 pi
// (k d mod n) / n, reduced in FP64 as the kernel does.
void delay_phase(size_t k, double d, size_t n, double* c, double* s) {
    const double r = std::fmod((double)k * d, (double)n);
    const double a = -2.0 * M_PI * r / (double)n;
    *c = std::cos(a);
    *s = std::sin(a);
}

std::mutex g_reg_mu;
std::vector<Builtin> g_reg;

int lookup(const std::string& name) {
    for (size_t i = 0; i < g_reg.size(); i++)
        if (g_reg[i].name == name) return (int)i;
    return -1;
}

// ---- reader ----------------------------------------------------------------

struct Node {
    bool list = false;
    std::string head;                  // list: operator symbol
    std::string atom;                  // atom: symbol text
    bool number = false;
    double value = 0;
    std::vector<std::unique_ptr<Node>> kids;
    std::vector<std::pair<std::string, std::unique_ptr<Node>>> kw;
    const Node* kwarg(const char* k) const {
        for (auto& p : kw)
            if (p.first == k) return p.second.get();
        return nullptr;
    }
};

struct Reader {
    const char* s;
    size_t i = 0, n;
    std::string err;
    explicit Reader(const char* src) : s(src), n(strlen(src)) {}
    void ws() {
        while (i < n) {
            if (isspace((unsigned char)s[i])) i++;
            else if (s[i] == ';') while (i < n && s[i] != '\n') i++;
            else break;
        }
    }
    static bool symch(char c) { return isalnum((unsigned char)c) || c == '-' || c == '_' || c == '?' || c == '*'; }
    std::string sym() {
        size_t b = i;
        while (i < n && symch(s[i])) i++;
        return std::string(s + b, i - b);
    }
    std::unique_ptr<Node> expr() {
        ws();
        if (i >= n) { err = "unexpected end of input"; return nullptr; }
        auto nd = std::make_unique<Node>();
        if (s[i] == '(') {
            i++;
            ws();
            if (i >= n || !(isalpha((unsigned char)s[i]) || s[i] == '-' || s[i] == '_' || s[i] == ':')) {
                err = "expected symbol after '('";
                return nullptr;
            }
            if (s[i] == ':') i++;
            nd->list = true;
            nd->head = sym();
            for (;;) {
                ws();
                if (i >= n) { err = "unexpected EOF"; return nullptr; }
                if (s[i] == ')') { i++; break; }
                if (s[i] == ':') {
                    i++;
                    std::string k = sym();
                    ws();
                    std::unique_ptr<Node> v;
                    if (i >= n || s[i] == ')' || s[i] == ':') {
                        v = std::make_unique<Node>();  // bare flag
                        v->atom = "true";
                        v->number = true;
                        v->value = 1;
                    } else {
                        v = expr();
                        if (!v) return nullptr;
                    }
                    nd->kw.emplace_back(k, std::move(v));
                } else {
                    auto c = expr();
                    if (!c) return nullptr;
                    nd->kids.push_back(std::move(c));
                }
            }
            return nd;
        }
        if (isdigit((unsigned char)s[i]) ||
            (s[i] == '-' && i + 1 < n && (isdigit((unsigned char)s[i + 1]) || s[i + 1] == '.'))) {
            char* end = nullptr;
            nd->number = true;
            nd->value = strtod(s + i, &end);
            nd->atom = std::string(s + i, end - (s + i));
            i = end - s;
            return nd;
        }
        if (isalpha((unsigned char)s[i]) || s[i] == '-' || s[i] == '_' || s[i] == '*') {
            nd->atom = sym();
            return nd;
        }
        err = std::string("unexpected character '") + s[i] + "'";
        return nullptr;
    }
};

const char* name_of(const Node* n) {
    if (!n) return nullptr;
    if (!n->list) return n->atom.c_str();
    return nullptr;
}

int parse_layout(const Node* n, faf_layout* out) {
    const char* s = name_of(n);
    if (!s) return -1;
    if (!strcmp(s, "hermitian")) *out = FAF_LAYOUT_HERMITIAN;
    else if (!strcmp(s, "interleaved")) *out = FAF_LAYOUT_INTERLEAVED;
    else if (!strcmp(s, "split")) *out = FAF_LAYOUT_SPLIT;
    else if (!strcmp(s, "real")) *out = FAF_LAYOUT_REAL;
    else if (!strcmp(s, "default")) *out = FAF_LAYOUT_DEFAULT;
    else return -1;
    return 0;
}

int parse_norm(const Node* n, faf_norm* out) {
    const char* s = name_of(n);
    if (!s) return -1;
    if (!strcmp(s, "none")) *out = FAF_NORM_NONE;
    else if (!strcmp(s, "ortho")) *out = FAF_NORM_ORTHO;
    else if (!strcmp(s, "forward")) *out = FAF_NORM_FORWARD;
    else if (!strcmp(s, "lazy")) *out = FAF_NORM_LAZY;
    else if (!strcmp(s, "jpeg2000")) *out = FAF_NORM_JPEG2000;
    else if (!strcmp(s, "default")) *out = FAF_NORM_DEFAULT;
    else return -1;
    return 0;
}

size_t size_of(const Node* nd) {
    const Node* sz = nd->kwarg("size");
    if (sz && sz->number) return (size_t)sz->value;
    if (!nd->kids.empty() && nd->kids[0]->number) return (size_t)nd->kids[0]->value;
    return 64;
}

int parse_precision(const Node* nd, faf_config& c, const char* form) {
    const Node* p = nd->kwarg("precision");
    if (!p) return 0;
    const char* s = name_of(p);
    if (s && !strcmp(s, "f32")) { c.precision = FAF_PREC_FP32; return 0; }
    if (s && !strcmp(s, "f64")) { c.precision = FAF_PREC_FP64; return 0; }
    fail("Chirp: (%s) :precision must be f32 or f64", form);
    return -1;
}

int parse_backend(const Node* nd, faf_config& c) {
    const Node* b = nd->kwarg("backend");
    if (!b) return 0;
    const char* s = name_of(b);
    if (s && (!strcmp(s, "cuda") || !strcmp(s, "auto"))) { c.backend = FAF_BACKEND_CUDA; return 0; }
    fail("Chirp: :backend must be cuda or auto");
    return -1;
}

// (rfft ...) / (irfft ...): reference src/chirp.c:1642-1686.
faf_transform* compile_rfft(const Node* nd, bool inverse) {
    faf_config c = faf_config_init(size_of(nd));
    if (inverse) c.dir = FAF_DIR_INVERSE;
    if (const Node* nn = nd->kwarg("norm")) {
        if (parse_norm(nn, &c.norm) != 0) { fail("Chirp: unknown :norm for rfft"); return nullptr; }
    }
    if (c.norm == FAF_NORM_JPEG2000 || c.norm == FAF_NORM_LAZY) {
        fail("Chirp: :norm jpeg2000/lazy is not valid on (rfft); use none|ortho|forward");
        return nullptr;
    }
    if (const Node* l = nd->kwarg("layout")) {
        if (parse_layout(l, &c.layout) != 0) { fail("Chirp: unknown :layout for rfft"); return nullptr; }
    }
    if (parse_precision(nd, c, "rfft") || parse_backend(nd, c)) return nullptr;
    if (nd->kwarg("bluestein")) {
        fail("Chirp: (rfft) does not support :bluestein; use (fft :bluestein) on a real buffer");
        return nullptr;
    }
    return faf_create_rfft(&c);
}

// (fft ...) / (ifft ...): reference src/chirp.c:1688-1727 (INTERLEAVED default).
faf_transform* compile_fft(const Node* nd, bool inverse) {
    faf_config c = faf_config_init(size_of(nd));
    c.layout = FAF_LAYOUT_INTERLEAVED;
    if (inverse) c.dir = FAF_DIR_INVERSE;
    if (const Node* nn = nd->kwarg("norm")) {
        if (parse_norm(nn, &c.norm) != 0) { fail("Chirp: unknown :norm for fft"); return nullptr; }
    }
    if (const Node* l = nd->kwarg("layout")) {
        if (parse_layout(l, &c.layout) != 0) { fail("Chirp: unknown :layout for fft"); return nullptr; }
    }
    if (parse_precision(nd, c, "fft") || parse_backend(nd, c)) return nullptr;
    if (nd->kwarg("bluestein")) c.flags |= FAF_FLAG_BLUESTEIN;
    if (nd->kwarg("measure")) c.flags |= FAF_FLAG_MEASURE;
    return faf_create_fft(&c);
}

bool is_spectral_op(const Node* n) {
    if (n->list) {
        if (n->head == "spectral" || n->head == "bandpass" || n->head == "mul-spectrum" ||
            n->head == "conj")
            return true;
        if (n->head == "custom" && !n->kids.empty() && !n->kids[0]->list) {
            const int idx = lookup(n->kids[0]->atom);
            return idx >= 0;
        }
        return false;
    }
    if (n->atom == "conj" || n->atom == "mul-spectrum") return true;
    return lookup(n->atom) >= 0;
}

int emit_op(const Node* n, faf_inst* out) {
    memset(out, 0, sizeof *out);
    out->packed = FAF_CALL_BUILTIN;
    const std::string h = n->list ? n->head : n->atom;
    if (h == "conj") { out->a0 = CHIRP_OP_CONJ; return 0; }
    if (h == "mul-spectrum") { out->a0 = CHIRP_OP_MUL; return 0; }
    if (h == "bandpass") {
        const Node* lo = n->kwarg("lo");
        const Node* hi = n->kwarg("hi");
        out->a0 = CHIRP_OP_BANDPASS;
        out->a1 = (uint32_t)(lo && lo->number ? (long)lo->value : 0);
        out->a2 = (uint32_t)(hi && hi->number ? (long)hi->value : 0);
        return 0;
    }
    std::string name;
    if (n->list && n->head == "spectral") {
        if (const Node* nm = n->kwarg("name")) name = nm->atom;
        else if (!n->kids.empty()) name = n->kids[0]->atom;
    } else if (n->list && n->head == "custom" && !n->kids.empty()) {
        name = n->kids[0]->atom;
    } else {
        name = h;
    }
    if (name.empty()) return fail("Chirp: spectral form needs a registered name");
    const int idx = lookup(name);
    if (idx < 0) return fail("Chirp: unknown spectral builtin '%s'", name.c_str());
    out->a0 = (uint32_t)idx;
    return 0;
}

faf_transform* compile_pipeline(const Node* p) {
    const auto& k = p->kids;
    if (k.empty() || !k[0]->list || k[0]->head != "rfft") return nullptr;
    const Node* head = k[0].get();
    const Node* tail = k.size() >= 2 ? k.back().get() : nullptr;
    bool has_inv = tail && tail->list && (tail->head == "irfft" || tail->head == "inverse");
    const size_t m0 = 1, m1 = has_inv ? k.size() - 1 : k.size();
    for (size_t i = m0; i < m1; i++)
        if (!is_spectral_op(k[i].get())) {
            fail("Chirp: fused rfft pipeline only accepts spectral/conj/mul-spectrum/bandpass "
                 "in the middle");
            return nullptr;
        }
    // Validate the whole form before any device plan is built.
    const size_t nops = m1 - m0;
    if (nops > (size_t)fafk::kMaxOps) {
        fail("Chirp: at most %d spectral ops per fused pipeline", fafk::kMaxOps);
        return nullptr;
    }
    std::vector<faf_inst> code(nops);
    for (size_t i = 0; i < nops; i++)
        if (emit_op(k[m0 + i].get(), &code[i]) != 0) return nullptr;
    if (has_inv && tail->head == "inverse" && tail->kwarg("size")) {
        fail("Chirp: (inverse) inherits size from the forward transform; delete :size "
             "(inherited)");
        return nullptr;
    }
    faf_transform* fwd = compile_rfft(head, false);
    if (!fwd) return nullptr;
    if (fwd->cfg.precision != FAF_PREC_FP32) {
        fail("Chirp: the fused pipeline runs in FP32 on the CUDA backend (:precision f64 is "
             "available for standalone (fft) / (rfft) forms)");
        faf_destroy_transform(fwd);
        return nullptr;
    }
    faf_transform* inv = nullptr;
    if (has_inv) {
        if (tail->head == "inverse") {
            faf_config ic = faf_config_inverse(fwd->cfg);
            inv = faf_create_rfft(&ic);
        } else if (!tail->kwarg("size") && tail->kids.empty()) {
            faf_config ic = faf_config_inverse(fwd->cfg);
            inv = faf_create_rfft(&ic);
        } else {
            inv = compile_rfft(tail, true);
        }
        if (!inv) {
            faf_destroy_transform(fwd);
            return nullptr;
        }
        if (inv->n != fwd->n) {
            fail("Chirp: (irfft) size %zu does not match (rfft) size %zu", inv->n, fwd->n);
            faf_destroy_transform(fwd);
            faf_destroy_transform(inv);
            return nullptr;
        }
    }
    faf_transform* t = alloc_transform();
    if (!t) {
        faf_destroy_transform(fwd);
        faf_destroy_transform(inv);
        return nullptr;
    }
    t->type = FAF_TRANSFORM_PIPELINE;
    t->n = fwd->n;
    t->precision = fwd->precision;
    t->inner = fwd;
    t->inner_inv = inv;
    t->cfg = fwd->cfg;
    t->cfg.layout = has_inv ? FAF_LAYOUT_REAL : fwd->cfg.layout;
    if (const Node* play = p->kwarg("layout")) {
        faf_layout lay;
        if (parse_layout(play, &lay) != 0) {
            fail("Chirp: unknown :layout for pipeline");
            faf_destroy_transform(t);
            return nullptr;
        }
        if (has_inv && lay != FAF_LAYOUT_DEFAULT)
            t->cfg.layout = lay == FAF_LAYOUT_INTERLEAVED ? FAF_LAYOUT_REAL : lay;
        else if (!has_inv && lay != FAF_LAYOUT_DEFAULT)
            t->cfg.layout = lay;
    }
    t->cfg.dir = has_inv ? FAF_DIR_INVERSE : FAF_DIR_FORWARD;
    t->flags = FAF_FLAG_REAL;
    if (nops) {
        t->code = (faf_inst*)calloc(nops, sizeof(faf_inst));
        t->n_inst = nops;
        memcpy(t->code, code.data(), nops * sizeof(faf_inst));
    }
    // One fused kernel: forward norm of the R2C, inverse norm of the C2R.
    const faf_norm fn = fwd->cfg.norm;
    const faf_norm in = inv ? inv->cfg.norm : FAF_NORM_NONE;
    std::string err;
    fafp::DevicePlan* dp = fafp::plan_pipeline((int)t->n, norm_scale(fn, false, t->n),
                                               inv ? norm_scale(in, true, t->n) : 1.0f, err);
    if (!dp) {
        fail("CUDA plan for pipeline n=%zu: %s", t->n, err.c_str());
        faf_destroy_transform(t);
        return nullptr;
    }
    t->device_plan = dp;
    return t;
}

}  // namespace

// ---- public registry API ---------------------------------------------------

extern "C" int chirp_register_spectral_ex(const char* name, chirp_spectral_fn f32,
                                          chirp_spectral_fn_f64 f64, void* ctx) {
    if (!name || !f32) return -1;
    std::lock_guard<std::mutex> lk(g_reg_mu);
    int idx = lookup(name);
    if (idx < 0) {
        g_reg.push_back(Builtin());
        idx = (int)g_reg.size() - 1;
        g_reg[idx].name = name;
    }
    g_reg[idx].f32 = f32;
    g_reg[idx].f64 = f64;
    g_reg[idx].kind = CHIRP_KIND_SPECTRAL;
    g_reg[idx].ctx = ctx;
    g_reg[idx].device = false;
    return idx;
}

extern "C" int chirp_register_spectral_device(const char* name, chirp_device_op op, double p0) {
    if (!name || !*name) {
        fail("chirp_register_spectral_device: name is required");
        return -1;
    }
    if ((int)op < CHIRP_DEVICE_GAIN || (int)op > CHIRP_DEVICE_HIGHPASS) {
        fail("chirp_register_spectral_device: unknown op %d", (int)op);
        return -1;
    }
    if (!std::isfinite(p0) || ((op == CHIRP_DEVICE_LOWPASS || op == CHIRP_DEVICE_HIGHPASS) && p0 < 0)) {
        fail("chirp_register_spectral_device: bad parameter %g for op %d", p0, (int)op);
        return -1;
    }
    std::lock_guard<std::mutex> lk(g_reg_mu);
    int idx = lookup(name);
    if (idx < 0) {
        g_reg.push_back(Builtin());
        idx = (int)g_reg.size() - 1;
        g_reg[idx].name = name;
    }
    Builtin& b = g_reg[idx];
    b.f32 = nullptr;
    b.f64 = nullptr;
    b.ctx = nullptr;
    b.kind = CHIRP_KIND_SPECTRAL;
    b.device = true;
    b.dop = (int)op;
    b.p0 = p0;
    return idx;
}

extern "C" int chirp_register_spectral(const char* name, chirp_spectral_fn fn, void* ctx) {
    return chirp_register_spectral_ex(name, fn, nullptr, ctx);
}

extern "C" int chirp_builtin_kind(int idx) {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    return (idx >= 0 && idx < (int)g_reg.size()) ? g_reg[idx].kind : CHIRP_KIND_OTHER;
}

extern "C" void* chirp_builtin_ctx(int idx) {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    return (idx >= 0 && idx < (int)g_reg.size()) ? g_reg[idx].ctx : nullptr;
}

extern "C" const char* chirp_builtin_name(int idx) {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    return (idx >= 0 && idx < (int)g_reg.size()) ? g_reg[idx].name.c_str() : nullptr;
}

extern "C" int chirp_count(void) {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    return (int)g_reg.size();
}

extern "C" void chirp_cleanup(void) {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_reg.clear();
}

extern "C" int chirp_bind(faf_transform* t, const char* name, void* re, void* im, size_t n_bins) {
    if (!t || !name || !re) {
        fail("chirp_bind: transform, name, and re are required");
        return -1;
    }
    if (strcmp(name, "H") && strcmp(name, "mul-spectrum") && strcmp(name, "kernel")) {
        fail("chirp_bind: unknown slot '%s' (use \"H\")", name);
        return -1;
    }
    t->user_aux = re;
    t->user_aux_im = im;
    t->user_aux_n = n_bins;
    return 0;
}

// Host application of one op (reference src/chirp.c:421-471).
extern "C" void chirp_apply_split_f32(const faf_transform* t, uint32_t a0, uint32_t a1,
                                      uint32_t a2, float* re, float* im, size_t n) {
    if (!re || n == 0) return;
    if (a0 == CHIRP_OP_CONJ) {
        if (!im) return;
        for (size_t i = 0; i < n; i++) im[i] = -im[i];
        return;
    }
    if (a0 == CHIRP_OP_MUL) {
        if (!im || !t || !t->user_aux || !t->user_aux_im) return;
        const size_t m = t->user_aux_n < n ? t->user_aux_n : n;
        std::vector<float> hr(m), hi(m);
        // H may live on the device
        if (ptr_is_device(t->user_aux)) {
            cudaMemcpy(hr.data(), t->user_aux, m * sizeof(float), cudaMemcpyDeviceToHost);
            cudaMemcpy(hi.data(), t->user_aux_im, m * sizeof(float), cudaMemcpyDeviceToHost);
        } else {
            memcpy(hr.data(), t->user_aux, m * sizeof(float));
            memcpy(hi.data(), t->user_aux_im, m * sizeof(float));
        }
        faf_herm_mul_f32(re, im, re, im, hr.data(), hi.data(), m);
        return;
    }
    if (a0 == CHIRP_OP_BANDPASS) {
        if (!im) return;
        for (size_t i = 0; i < n; i++)
            if (i < a1 || i > a2) { re[i] = 0.f; im[i] = 0.f; }
        return;
    }
    Builtin b;
    {
        std::lock_guard<std::mutex> lk(g_reg_mu);
        if ((int)a0 < 0 || a0 >= g_reg.size()) return;
        b = g_reg[a0];
    }
    if (b.device) {  // the device op's math, on host bins (FP64 phases)
        if (!im) return;
        const size_t len = t ? t->n : 2 * (n - 1);
        for (size_t k = 0; k < n; k++) {
            double c = 1, s = 0, g = 1;
            if (b.dop == CHIRP_DEVICE_GAIN) g = b.p0;
            else if (b.dop == CHIRP_DEVICE_PHASE) { c = std::cos(b.p0); s = std::sin(b.p0); }
            else if (b.dop == CHIRP_DEVICE_DELAY) delay_phase(k, b.p0, len, &c, &s);
            else if (b.dop == CHIRP_DEVICE_LOWPASS) g = (double)k > b.p0 ? 0.0 : 1.0;
            else if (b.dop == CHIRP_DEVICE_HIGHPASS) g = (double)k < b.p0 ? 0.0 : 1.0;
            const double r = re[k], i = im[k];
            re[k] = (float)(g * (r * c - i * s));
            im[k] = (float)(g * (r * s + i * c));
        }
        return;
    }
    if (!b.f32 || !im) return;
    b.f32(re, im, n, b.ctx);
    if (b.kind == CHIRP_KIND_HERMITIAN) {
        im[0] = 0.f;
        im[n - 1] = 0.f;
    }
}

extern "C" faf_transform* chirp_compile(const char* source) {
    if (!source) return nullptr;
    Reader rd(source);
    // A program is one or more top-level forms; the last one is the body.
    std::vector<std::unique_ptr<Node>> forms;
    for (;;) {
        rd.ws();
        if (rd.i >= rd.n) break;
        auto f = rd.expr();
        if (!f) {
            fail("Chirp: failed to parse program (%s)", rd.err.c_str());
            return nullptr;
        }
        forms.push_back(std::move(f));
    }
    if (forms.empty()) {
        fail("Chirp: failed to parse program (empty)");
        return nullptr;
    }
    const Node* main = forms.back().get();
    if (!main->list) {
        fail("Chirp: program body must be a form");
        return nullptr;
    }
    if (main->head == "rfft") return compile_rfft(main, false);
    if (main->head == "irfft") return compile_rfft(main, true);
    if (main->head == "fft") return compile_fft(main, false);
    if (main->head == "ifft") return compile_fft(main, true);
    if (main->head == "pipeline") {
        if (main->kids.size() == 1 && main->kids[0]->list) {
            const Node* c0 = main->kids[0].get();
            if (c0->head == "rfft") return compile_rfft(c0, false);
            if (c0->head == "irfft") return compile_rfft(c0, true);
            if (c0->head == "fft") return compile_fft(c0, false);
            if (c0->head == "ifft") return compile_fft(c0, true);
        }
        if (!main->kids.empty() && main->kids[0]->list && main->kids[0]->head == "rfft")
            return compile_pipeline(main);
        for (auto& c : main->kids)
            if (c->list && (c->head == "rfft" || c->head == "irfft")) {
                fail("Chirp: (rfft)/(irfft) must lead a fused pipeline (rfft ... irfft); they "
                     "cannot mix with FFT IR stages");
                return nullptr;
            }
    }
    fail("Chirp: form '%s' is outside the CUDA transform path (fft, ifft, rfft, irfft, "
         "fused rfft pipeline)", main->head.c_str());
    return nullptr;
}

// ---- pipeline op resolution for the fused kernel -------------------------

namespace fafapi {

int resolve_pipeline_ops(const faf_transform* t, fafk::PipeOp* ops, int cap, bool* host_ops,
                         cudaStream_t st) {
    *host_ops = false;
    const size_t nb = t->n / 2 + 1;
    int k = 0;
    for (size_t i = 0; i < t->n_inst; i++) {
        const faf_inst& in = t->code[i];
        fafk::PipeOp op;
        memset(&op, 0, sizeof op);
        if (in.a0 == CHIRP_OP_CONJ) {
            op.code = fafk::OP_CONJ;
        } else if (in.a0 == CHIRP_OP_BANDPASS) {
            op.code = fafk::OP_BANDPASS;
            op.lo = (int)std::min<uint32_t>(in.a1, 0x7fffffff);
            op.hi = (int)std::min<uint32_t>(in.a2, 0x7fffffff);
        } else if (in.a0 == CHIRP_OP_MUL) {
            if (!t->user_aux || !t->user_aux_im) continue;  // unbound: no-op, as the reference
            const size_t m = std::min(t->user_aux_n, nb);
            if (m == 0) continue;
            op.code = fafk::OP_MUL;
            op.m = (int)m;
            if (ptr_is_device(t->user_aux) && ptr_is_device(t->user_aux_im)) {
                op.hr = (const float*)t->user_aux;
                op.hi_ = (const float*)t->user_aux_im;
            } else {
                // Host H: copied to a plan buffer on every execute (H is read
                // live, like the reference, so later edits are honoured).
                fafp::DevicePlan* p = plan_of(t);
                std::lock_guard<std::mutex> lk(p->scratch_mu);
                const size_t bytes = 2 * nb * sizeof(float);
                if (p->scratch_bytes < bytes) {
                    cudaFree(p->d_scratch);
                    p->d_scratch = nullptr;
                    p->scratch_bytes = 0;
                    cudaError_t e = cudaMalloc(&p->d_scratch, bytes);
                    if (e != cudaSuccess) return cuda_fail(e, "bound spectrum upload");
                    p->scratch_bytes = bytes;
                }
                float* dh = (float*)p->d_scratch;
                cudaError_t e = cudaMemcpyAsync(dh, t->user_aux, m * sizeof(float),
                                                cudaMemcpyHostToDevice, st);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(dh + nb, t->user_aux_im, m * sizeof(float),
                                        cudaMemcpyHostToDevice, st);
                if (e != cudaSuccess) return cuda_fail(e, "bound spectrum upload");
                op.hr = dh;
                op.hi_ = dh + nb;
            }
        } else {
            Builtin b;
            {
                std::lock_guard<std::mutex> lk(g_reg_mu);
                if (in.a0 < g_reg.size()) b = g_reg[in.a0];
            }
            if (!b.device) {
                *host_ops = true;  // a registered host callback
                continue;
            }
            switch (b.dop) {
            case CHIRP_DEVICE_GAIN:
                op.code = fafk::OP_SCALE;
                op.f0 = (float)b.p0;
                break;
            case CHIRP_DEVICE_PHASE:
                op.code = fafk::OP_ROTATE;
                op.f0 = (float)std::cos(b.p0);
                op.f1 = (float)std::sin(b.p0);
                break;
            case CHIRP_DEVICE_DELAY:
                op.code = fafk::OP_DELAY;
                op.d0 = b.p0;
                op.n = (int)t->n;
                break;
            case CHIRP_DEVICE_LOWPASS:
                op.code = fafk::OP_BANDPASS;
                op.lo = 0;
                op.hi = (int)std::min(std::floor(b.p0), 2147483647.0);
                break;
            default:  // CHIRP_DEVICE_HIGHPASS
                op.code = fafk::OP_BANDPASS;
                op.lo = (int)std::min(std::ceil(b.p0), 2147483647.0);
                op.hi = 0x7fffffff;
                break;
            }
        }
        if (k >= cap) return fail("too many pipeline ops");
        ops[k++] = op;
    }
    return k;
}

void apply_ops_host(const faf_transform* t, float* re, float* im, size_t nb) {
    for (size_t i = 0; i < t->n_inst; i++) {
        const faf_inst& in = t->code[i];
        chirp_apply_split_f32(t, in.a0, in.a1, in.a2, re, im, nb);
    }
}

}  // namespace fafapi
