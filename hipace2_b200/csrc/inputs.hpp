// Input-file store and math-expression compiler for the quasi-static slice loop.
//
// The reference reads its parameters with amrex::ParmParse (`key = v1 v2 ...`, `#` comments,
// later keys and command-line `key=value` overrides win) and evaluates every numeric value as a
// math expression with user constants from `my_constants.*` (utils/Parser.H:37-51, 316-395).
// This header restates that interface: `InputStore` holds the key/value table, and `Expr` is a
// compiled expression (postfix byte code, fixed capacity, trivially copyable) that host code and
// CUDA kernels evaluate with the same `eval` routine, e.g. the plasma density profile
// `plasma.density(x,y,z) = 1+0.05*(x*x+y*y)`.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef __CUDACC__
#define HPQ_HD __host__ __device__
#else
#define HPQ_HD
#endif

namespace hpq {

struct InputError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// ---------------------------------------------------------------------------------------------
// Compiled expression
// ---------------------------------------------------------------------------------------------
enum ExprOp : uint8_t {
    OP_CONST = 0, OP_VAR, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_POW, OP_NEG,
    OP_LT, OP_GT, OP_LE, OP_GE, OP_EQ, OP_NE, OP_AND, OP_OR,
    OP_SQRT, OP_EXP, OP_LOG, OP_LOG10, OP_SIN, OP_COS, OP_TAN, OP_ASIN, OP_ACOS, OP_ATAN,
    OP_SINH, OP_COSH, OP_TANH, OP_ABS, OP_FLOOR, OP_CEIL, OP_HEAVISIDE,
    OP_ATAN2, OP_MIN, OP_MAX, OP_FMOD, OP_IF
};

struct Expr {
    static constexpr int kMaxOps = 96;
    static constexpr int kMaxStack = 24;
    int nops = 0;
    int nvars = 0;
    uint8_t op[kMaxOps] = {};
    uint8_t arg[kMaxOps] = {};     // variable index for OP_VAR
    double cst[kMaxOps] = {};      // value for OP_CONST

    HPQ_HD double eval(const double* v) const {
        double st[kMaxStack];
        int sp = 0;
        for (int k = 0; k < nops; ++k) {
            const int o = op[k];
            if (o == OP_CONST) { st[sp++] = cst[k]; continue; }
            if (o == OP_VAR) { st[sp++] = v[arg[k]]; continue; }
            if (o == OP_NEG) { st[sp - 1] = -st[sp - 1]; continue; }
            if (o >= OP_SQRT && o <= OP_HEAVISIDE) {
                double a = st[sp - 1], r = 0;
                switch (o) {
                    case OP_SQRT: r = sqrt(a); break;
                    case OP_EXP: r = exp(a); break;
                    case OP_LOG: r = log(a); break;
                    case OP_LOG10: r = log10(a); break;
                    case OP_SIN: r = sin(a); break;
                    case OP_COS: r = cos(a); break;
                    case OP_TAN: r = tan(a); break;
                    case OP_ASIN: r = asin(a); break;
                    case OP_ACOS: r = acos(a); break;
                    case OP_ATAN: r = atan(a); break;
                    case OP_SINH: r = sinh(a); break;
                    case OP_COSH: r = cosh(a); break;
                    case OP_TANH: r = tanh(a); break;
                    case OP_ABS: r = fabs(a); break;
                    case OP_FLOOR: r = floor(a); break;
                    case OP_CEIL: r = ceil(a); break;
                    case OP_HEAVISIDE: r = a > 0 ? 1.0 : (a < 0 ? 0.0 : 0.5); break;
                    default: break;
                }
                st[sp - 1] = r;
                continue;
            }
            if (o == OP_IF) {
                double c = st[sp - 3], a = st[sp - 2], b = st[sp - 1];
                sp -= 2;
                st[sp - 1] = (c != 0.0) ? a : b;
                continue;
            }
            double b = st[--sp];
            double a = st[sp - 1];
            double r = 0;
            switch (o) {
                case OP_ADD: r = a + b; break;
                case OP_SUB: r = a - b; break;
                case OP_MUL: r = a * b; break;
                case OP_DIV: r = a / b; break;
                case OP_POW: r = pow(a, b); break;
                case OP_LT: r = a < b; break;
                case OP_GT: r = a > b; break;
                case OP_LE: r = a <= b; break;
                case OP_GE: r = a >= b; break;
                case OP_EQ: r = a == b; break;
                case OP_NE: r = a != b; break;
                case OP_AND: r = (a != 0.0) && (b != 0.0); break;
                case OP_OR: r = (a != 0.0) || (b != 0.0); break;
                case OP_ATAN2: r = atan2(a, b); break;
                case OP_MIN: r = a < b ? a : b; break;
                case OP_MAX: r = a > b ? a : b; break;
                case OP_FMOD: r = fmod(a, b); break;
                default: break;
            }
            st[sp - 1] = r;
        }
        return sp > 0 ? st[0] : 0.0;
    }
    bool is_constant() const {
        for (int k = 0; k < nops; ++k) if (op[k] == OP_VAR) return false;
        return true;
    }
};

// Recursive-descent compiler: expression string -> postfix program.
// Grammar (lowest to highest precedence): or, and, comparison, +/-, * /, unary -, ^ (right assoc).
class ExprCompiler {
public:
    ExprCompiler(const std::string& s, const std::vector<std::string>& vars,
                 const std::map<std::string, double>& consts)
        : s_(s), vars_(vars), consts_(consts) {}

    Expr compile() {
        pos_ = 0;
        parse_or();
        skip();
        if (pos_ != s_.size()) fail("unexpected character '" + std::string(1, s_[pos_]) + "'");
        int depth = 0, maxdepth = 0;
        for (int k = 0; k < e_.nops; ++k) {
            const int o = e_.op[k];
            if (o == OP_CONST || o == OP_VAR) depth++;
            else if (o == OP_NEG || (o >= OP_SQRT && o <= OP_HEAVISIDE)) {}
            else if (o == OP_IF) depth -= 2;
            else depth -= 1;
            if (depth > maxdepth) maxdepth = depth;
        }
        if (maxdepth > Expr::kMaxStack) fail("expression too deeply nested");
        e_.nvars = (int)vars_.size();
        return e_;
    }

private:
    const std::string s_;
    const std::vector<std::string> vars_;
    const std::map<std::string, double>& consts_;
    size_t pos_ = 0;
    Expr e_;

    [[noreturn]] void fail(const std::string& m) {
        throw InputError("cannot parse expression '" + s_ + "': " + m);
    }
    void emit(uint8_t o, double c = 0.0, uint8_t a = 0) {
        if (e_.nops >= Expr::kMaxOps) fail("expression too long");
        e_.op[e_.nops] = o; e_.cst[e_.nops] = c; e_.arg[e_.nops] = a; e_.nops++;
    }
    void skip() { while (pos_ < s_.size() && isspace((unsigned char)s_[pos_])) pos_++; }
    bool accept(const char* t) {
        skip();
        size_t n = strlen(t);
        if (s_.compare(pos_, n, t) == 0) { pos_ += n; return true; }
        return false;
    }
    void parse_or() {
        parse_and();
        while (accept("||")) { parse_and(); emit(OP_OR); }
    }
    void parse_and() {
        parse_cmp();
        while (accept("&&")) { parse_cmp(); emit(OP_AND); }
    }
    void parse_cmp() {
        parse_add();
        for (;;) {
            if (accept("<=")) { parse_add(); emit(OP_LE); }
            else if (accept(">=")) { parse_add(); emit(OP_GE); }
            else if (accept("==")) { parse_add(); emit(OP_EQ); }
            else if (accept("!=")) { parse_add(); emit(OP_NE); }
            else if (accept("<")) { parse_add(); emit(OP_LT); }
            else if (accept(">")) { parse_add(); emit(OP_GT); }
            else break;
        }
    }
    void parse_add() {
        parse_mul();
        for (;;) {
            if (accept("+")) { parse_mul(); emit(OP_ADD); }
            else if (accept("-")) { parse_mul(); emit(OP_SUB); }
            else break;
        }
    }
    void parse_mul() {
        parse_unary();
        for (;;) {
            skip();
            if (s_.compare(pos_, 2, "**") == 0) break;  // handled in parse_pow
            if (accept("*")) { parse_unary(); emit(OP_MUL); }
            else if (accept("/")) { parse_unary(); emit(OP_DIV); }
            else break;
        }
    }
    void parse_unary() {
        if (accept("-")) { parse_unary(); emit(OP_NEG); return; }
        if (accept("+")) { parse_unary(); return; }
        parse_pow();
    }
    void parse_pow() {
        parse_atom();
        if (accept("^") || accept("**")) { parse_unary(); emit(OP_POW); }
    }
    void parse_atom() {
        skip();
        if (pos_ >= s_.size()) fail("unexpected end");
        char c = s_[pos_];
        if (c == '(') {
            pos_++;
            parse_or();
            if (!accept(")")) fail("missing ')'");
            return;
        }
        if (isdigit((unsigned char)c) || c == '.') {
            const char* b = s_.c_str() + pos_;
            char* e = nullptr;
            double v = strtod(b, &e);
            if (e == b) fail("bad number");
            pos_ += (size_t)(e - b);
            emit(OP_CONST, v);
            return;
        }
        if (isalpha((unsigned char)c) || c == '_') {
            size_t b = pos_;
            while (pos_ < s_.size() && (isalnum((unsigned char)s_[pos_]) || s_[pos_] == '_')) pos_++;
            std::string id = s_.substr(b, pos_ - b);
            skip();
            if (pos_ < s_.size() && s_[pos_] == '(') {
                pos_++;
                int nargs = 0;
                skip();
                if (!accept(")")) {
                    for (;;) {
                        parse_or();
                        nargs++;
                        if (accept(",")) continue;
                        if (accept(")")) break;
                        fail("expected ',' or ')' in call of " + id);
                    }
                }
                call(id, nargs);
                return;
            }
            for (size_t k = 0; k < vars_.size(); ++k) {
                if (vars_[k] == id) { emit(OP_VAR, 0.0, (uint8_t)k); return; }
            }
            auto it = consts_.find(id);
            if (it != consts_.end()) { emit(OP_CONST, it->second); return; }
            fail("unknown symbol '" + id + "'");
        }
        fail("unexpected character '" + std::string(1, c) + "'");
    }
    void call(const std::string& f, int n) {
        static const std::map<std::string, uint8_t> unary = {
            {"sqrt", OP_SQRT}, {"exp", OP_EXP}, {"log", OP_LOG}, {"log10", OP_LOG10},
            {"sin", OP_SIN}, {"cos", OP_COS}, {"tan", OP_TAN}, {"asin", OP_ASIN},
            {"acos", OP_ACOS}, {"atan", OP_ATAN}, {"sinh", OP_SINH}, {"cosh", OP_COSH},
            {"tanh", OP_TANH}, {"abs", OP_ABS}, {"fabs", OP_ABS}, {"floor", OP_FLOOR},
            {"ceil", OP_CEIL}, {"heaviside", OP_HEAVISIDE}};
        static const std::map<std::string, uint8_t> binary = {
            {"pow", OP_POW}, {"atan2", OP_ATAN2}, {"min", OP_MIN}, {"max", OP_MAX},
            {"fmod", OP_FMOD}};
        auto u = unary.find(f);
        if (u != unary.end()) { if (n != 1) fail(f + " takes 1 argument"); emit(u->second); return; }
        auto b = binary.find(f);
        if (b != binary.end()) { if (n != 2) fail(f + " takes 2 arguments"); emit(b->second); return; }
        if (f == "if") { if (n != 3) fail("if takes 3 arguments"); emit(OP_IF); return; }
        fail("unknown function '" + f + "'");
    }
};

// ---------------------------------------------------------------------------------------------
// Key/value store with ParmParse semantics
// ---------------------------------------------------------------------------------------------
class InputStore {
public:
    InputStore() = default;

    // Parse an input file text; later definitions of a key override earlier ones.
    void parse_text(const std::string& text) {
        std::string joined;
        // join continuation: a value may be quoted across spaces; lines are independent
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line)) parse_line(line);
    }
    // Command-line style override "key = v1 v2" or "key=v".
    void parse_line(std::string line) {
        auto hash = line.find('#');
        if (hash != std::string::npos) {
            // a '#' inside quotes is kept
            bool inq = false;
            size_t cut = std::string::npos;
            for (size_t i = 0; i < line.size(); ++i) {
                if (line[i] == '"') inq = !inq;
                if (line[i] == '#' && !inq) { cut = i; break; }
            }
            if (cut != std::string::npos) line = line.substr(0, cut);
        }
        auto eq = line.find('=');
        if (eq == std::string::npos) {
            for (char ch : line) if (!isspace((unsigned char)ch)) throw InputError("line without '=': " + line);
            return;
        }
        std::string key = trim(line.substr(0, eq));
        if (key.empty()) throw InputError("empty key in line: " + line);
        std::vector<std::string> vals = tokenize(line.substr(eq + 1));
        table_[key] = vals;
    }

    bool contains(const std::string& k) const { return table_.count(k) > 0; }
    const std::vector<std::string>& raw(const std::string& k) const {
        auto it = table_.find(k);
        if (it == table_.end()) throw InputError("missing required input '" + k + "'");
        used_.insert(k);
        return it->second;
    }
    std::vector<std::string> keys() const {
        std::vector<std::string> r;
        for (auto& kv : table_) r.push_back(kv.first);
        return r;
    }
    std::vector<std::string> unused_keys() const {
        std::vector<std::string> r;
        for (auto& kv : table_) if (!used_.count(kv.first)) r.push_back(kv.first);
        return r;
    }
    void mark_used(const std::string& k) const { used_.insert(k); }

    // Constants available to every expression: physical constants (SI, as the reference adds
    // them before reading the file) plus `my_constants.<name>`, evaluated in file order.
    std::map<std::string, double> constants() const {
        std::map<std::string, double> c = {
            {"pi", 3.14159265358979323846}, {"true", 1.0}, {"false", 0.0},
            {"clight", 299792458.0}, {"epsilon0", 8.8541878128e-12},
            {"mu0", 1.25663706212e-06}, {"q_e", 1.602176634e-19},
            {"m_e", 9.1093837015e-31}, {"m_p", 1.67262192369e-27},
            {"hbar", 1.054571817e-34}, {"r_e", 2.8179403262e-15}};
        // user constants may depend on one another; resolve iteratively
        std::vector<std::pair<std::string, std::string>> pending;
        for (auto& kv : table_) {
            if (kv.first.rfind("my_constants.", 0) == 0) {
                used_.insert(kv.first);
                std::string joined;
                for (auto& t : kv.second) joined += t + " ";
                pending.push_back({kv.first.substr(13), joined});
            }
        }
        for (int pass = 0; pass < 8 && !pending.empty(); ++pass) {
            std::vector<std::pair<std::string, std::string>> left;
            for (auto& p : pending) {
                try {
                    Expr e = ExprCompiler(p.second, {}, c).compile();
                    c[p.first] = e.eval(nullptr);
                } catch (const InputError&) {
                    left.push_back(p);
                }
            }
            pending.swap(left);
        }
        if (!pending.empty()) throw InputError("cannot resolve my_constants." + pending[0].first);
        return c;
    }

    // Typed queries (queryWithParser / getWithParser restated)
    bool query_expr_vec(const std::string& k, std::vector<double>& out) const {
        if (!contains(k)) return false;
        auto c = constants();
        out.clear();
        for (auto& t : raw(k)) out.push_back(ExprCompiler(t, {}, c).compile().eval(nullptr));
        return true;
    }
    // A scalar joins all tokens of the value with spaces before parsing (fillWithParserArr).
    template <class T>
    bool query(const std::string& k, T& v) const {
        std::string joined;
        if (!query_str(k, joined)) return false;
        double d = ExprCompiler(joined, {}, constants()).compile().eval(nullptr);
        v = (T)(std::is_integral<T>::value ? std::llround(d) : d);
        return true;
    }
    bool query_bool(const std::string& k, bool& v) const {
        if (!contains(k)) return false;
        auto& r = raw(k);
        if (r.size() != 1) throw InputError("input '" + k + "' expects one value");
        std::string s = r[0];
        if (s == "true" || s == "True") { v = true; return true; }
        if (s == "false" || s == "False") { v = false; return true; }
        double d;
        query(k, d);
        v = d != 0.0;
        return true;
    }
    template <class T, size_t N>
    bool query_arr(const std::string& k, T (&v)[N]) const {
        std::vector<double> d;
        if (!query_expr_vec(k, d)) return false;
        if (d.size() != N) throw InputError("input '" + k + "' expects " + std::to_string(N) + " values");
        for (size_t i = 0; i < N; ++i) v[i] = (T)(std::is_integral<T>::value ? std::llround(d[i]) : d[i]);
        return true;
    }
    template <class T>
    void get(const std::string& k, T& v) const {
        if (!query(k, v)) throw InputError("missing required input '" + k + "'");
    }
    template <class T, size_t N>
    void get_arr(const std::string& k, T (&v)[N]) const {
        if (!query_arr(k, v)) throw InputError("missing required input '" + k + "'");
    }
    bool query_str(const std::string& k, std::string& v) const {
        if (!contains(k)) return false;
        auto& r = raw(k);
        v.clear();
        for (size_t i = 0; i < r.size(); ++i) v += (i ? " " : "") + r[i];
        return true;
    }
    std::vector<std::string> query_strs(const std::string& k) const {
        if (!contains(k)) return {};
        return raw(k);
    }
    // Function of named variables, e.g. density(x,y,z)
    Expr function(const std::string& expr_text, const std::vector<std::string>& vars) const {
        return ExprCompiler(expr_text, vars, constants()).compile();
    }

private:
    std::map<std::string, std::vector<std::string>> table_;
    mutable std::set<std::string> used_;

    static std::string trim(const std::string& s) {
        size_t b = 0, e = s.size();
        while (b < e && isspace((unsigned char)s[b])) b++;
        while (e > b && isspace((unsigned char)s[e - 1])) e--;
        return s.substr(b, e - b);
    }
    static std::vector<std::string> tokenize(const std::string& s) {
        std::vector<std::string> r;
        size_t i = 0;
        while (i < s.size()) {
            while (i < s.size() && isspace((unsigned char)s[i])) i++;
            if (i >= s.size()) break;
            if (s[i] == '"') {
                size_t j = s.find('"', i + 1);
                if (j == std::string::npos) throw InputError("unterminated quote in: " + s);
                r.push_back(s.substr(i + 1, j - i - 1));
                i = j + 1;
            } else {
                size_t j = i;
                while (j < s.size() && !isspace((unsigned char)s[j])) j++;
                r.push_back(s.substr(i, j - i));
                i = j;
            }
        }
        return r;
    }
};

}  // namespace hpq
