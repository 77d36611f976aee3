// Expressions of x, y, z, t evaluated at every grid node on the device.
//
// The reference evaluates its LaTeX right sides, coefficients and boundary
// expressions node by node on the host (src/expression_eval.cpp:805-978, called
// per node from src/backends/cpu/solver.cpp:197 and cpu_utils.cpp:520-530).
// Here an expression is compiled once on the host into a postfix program and
// the program is run by one GPU thread per node. The language is the
// reference's: LaTeX commands turned into infix (ConvertLatexToInfix,
// expression_eval.cpp:179-387), letters-only identifiers lower-cased, implicit
// multiplication between adjacent primaries, '^' right-associative and taking
// a unary operand (so -\pi^2 is (-pi)^2, as in the reference), and the
// reference's guarded arithmetic (division by |d| < 1e-12, negative base with
// a non-integer exponent, tan/asin/acos/log/sqrt domains, exp clamped at
// +-700) giving the same NaN/inf/0 results. Transcendental functions are
// CUDA's on the device, so values can differ from the host C library in the
// last bits.
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "host.h"

namespace pdeb {

namespace {

constexpr int kExprMaxOps = 512;
constexpr int kExprMaxStack = 48;
constexpr int kExprMaxDepth = 100;     // parser nesting limit of the reference
constexpr double kExprDivEps = 1e-12;  // guarded division of the reference
constexpr double kExprPi = 3.14159265358979323846;
constexpr double kExprExpLimit = 700.0;

enum ExprOp : uint8_t {
  kNum, kX, kY, kZ, kT, kAdd, kSub, kMul, kDiv, kPow, kNeg,
  kSin, kCos, kTan, kSinh, kCosh, kTanh, kAsin, kAcos, kAtan, kExp, kLog, kSqrt,
  kFloor, kCeil, kRound, kAbs, kSign, kErf, kMin, kMax, kAtan2, kPow2,
  kZero1  // any other function name: its argument is evaluated, the value is 0
};

struct ExprProg {
  int n;
  int depth;
  uint8_t op[kExprMaxOps];
  double val[kExprMaxOps];
};

// ------------------------------------------------------------- evaluation

__host__ __device__ inline double expr_run(const ExprProg& P, double x, double y, double z, double t) {
  double st[kExprMaxStack];
  int sp = 0;
  const double qnan = nan("");
  for (int q = 0; q < P.n; ++q) {
    const int op = P.op[q];
    if (op <= kT) {
      st[sp++] = op == kNum ? P.val[q] : (op == kX ? x : (op == kY ? y : (op == kZ ? z : t)));
      continue;
    }
    if (op == kAdd || op == kSub || op == kMul || op == kDiv || op == kPow || op == kMin || op == kMax ||
        op == kAtan2 || op == kPow2) {
      const double b = st[--sp];
      const double a = st[sp - 1];
      double r;
      switch (op) {
        case kAdd: r = a + b; break;
        case kSub: r = a - b; break;
        case kMul: r = a * b; break;
        case kDiv:
          if (fabs(b) < kExprDivEps) {
            r = qnan;
          } else {
            r = a / b;
            if (!isfinite(r)) r = qnan;
          }
          break;
        case kPow:
          if (a < 0.0 && floor(b) != b) {
            r = qnan;
          } else {
            r = pow(a, b);
            if (!isfinite(r)) r = qnan;
          }
          break;
        case kMin: r = (b < a) ? b : a; break;
        case kMax: r = (a < b) ? b : a; break;
        case kAtan2: r = atan2(a, b); break;
        case kPow2: r = (a < 0.0 && floor(b) != b) ? qnan : pow(a, b); break;
        default: r = 0.0; break;
      }
      st[sp - 1] = r;
      continue;
    }
    const double v = st[sp - 1];
    double r;
    switch (op) {
      case kNeg: r = -v; break;
      case kSin: r = sin(v); break;
      case kCos: r = cos(v); break;
      case kTan: r = fabs(cos(v)) < kExprDivEps ? qnan : tan(v); break;
      case kSinh: r = sinh(v); break;
      case kCosh: r = cosh(v); break;
      case kTanh: r = tanh(v); break;
      case kAsin: r = (v < -1.0 || v > 1.0) ? qnan : asin(v); break;
      case kAcos: r = (v < -1.0 || v > 1.0) ? qnan : acos(v); break;
      case kAtan: r = atan(v); break;
      case kExp: r = v > kExprExpLimit ? HUGE_VAL : (v < -kExprExpLimit ? 0.0 : exp(v)); break;
      case kLog: r = v <= 0.0 ? qnan : log(v); break;
      case kSqrt: r = v < 0.0 ? qnan : sqrt(v); break;
      case kFloor: r = floor(v); break;
      case kCeil: r = ceil(v); break;
      case kRound: r = round(v); break;
      case kAbs: r = fabs(v); break;
      case kSign: r = v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); break;
      case kErf: r = erf(v); break;
      default: r = 0.0; break;
    }
    st[sp - 1] = r;
  }
  return sp > 0 ? st[sp - 1] : 0.0;
}

// Where the nodes of a launch sit: the launch walks an (na, nb, nc) index box
// (a fastest) and each coordinate is either base + index*step for one of the
// three indices (unfused, as the host computes min + i*h) or the fixed base.
struct NodeMap {
  int na, nb;
  int axis[3];     // 0, 1, 2: index a, b, c; 3: fixed at base
  double base[3];
  double step[3];
  int has_prog;    // 0: no expression, the linear form alone
  int linear;      // 1: non-finite values fall back to the linear form
  double lin[4];   // constant, x, y, z coefficients of the linear form
};

__device__ inline double node_coord(const NodeMap& m, int c, int a, int b, int k) {
  const int ax = m.axis[c];
  if (ax == 3) return m.base[c];
  const int idx = ax == 0 ? a : (ax == 1 ? b : k);
  return __dadd_rn(m.base[c], __dmul_rn(double(idx), m.step[c]));
}

__global__ void k_eval_expr(const ExprProg* __restrict__ prog, NodeMap m, long long n, double t,
                            double* __restrict__ out) {
  __shared__ ExprProg P;
  {
    const int* s = reinterpret_cast<const int*>(prog);
    int* d = reinterpret_cast<int*>(&P);
    for (int q = threadIdx.x; q < (int)(sizeof(ExprProg) / 4); q += blockDim.x) d[q] = s[q];
  }
  __syncthreads();
  for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < n;
       id += (long long)gridDim.x * blockDim.x) {
    const int a = int(id % m.na), b = int((id / m.na) % m.nb);
    const int k = int(id / ((long long)m.na * m.nb));
    const double x = node_coord(m, 0, a, b, k);
    const double y = node_coord(m, 1, a, b, k);
    const double z = node_coord(m, 2, a, b, k);
    double v = m.has_prog ? expr_run(P, x, y, z, t) : nan("");
    if (m.linear && !isfinite(v))
      v = __dadd_rn(__dadd_rn(__dadd_rn(m.lin[0], __dmul_rn(m.lin[1], x)), __dmul_rn(m.lin[2], y)),
                    __dmul_rn(m.lin[3], z));
    out[id] = v;
  }
}

// ------------------------------------------------------------ compilation

struct Failure {
  std::string what;
};

bool is_alpha(char c) { return std::isalpha(static_cast<unsigned char>(c)) != 0; }
bool is_space(char c) { return std::isspace(static_cast<unsigned char>(c)) != 0; }
std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower(static_cast<unsigned char>(c));
  return s;
}

// The text between a bracket and its match (nesting of the same bracket only).
std::string take_group(const std::string& in, size_t* at, char open, char close) {
  if (*at >= in.size() || in[*at] != open) throw Failure{std::string("expected '") + open + "'"};
  int depth = 0;
  for (size_t q = *at + 1; q < in.size(); ++q) {
    if (in[q] == open) {
      ++depth;
    } else if (in[q] == close) {
      if (depth == 0) {
        std::string g = in.substr(*at + 1, q - *at - 1);
        *at = q + 1;
        return g;
      }
      --depth;
    }
  }
  throw Failure{std::string("unterminated '") + open + "'"};
}

void skip_spaces(const std::string& in, size_t* at) {
  while (*at < in.size() && is_space(in[*at])) ++*at;
}

std::string to_infix(const std::string& in);

// One LaTeX command at `at` (a backslash) as infix text.
std::string command(const std::string& in, size_t* at) {
  size_t s = *at + 1, e = s;
  while (e < in.size() && is_alpha(in[e])) ++e;
  if (e == s) {
    if (e < in.size() && in[e] == ',') {  // thin space
      *at = e + 1;
      return "";
    }
    throw Failure{"invalid latex command"};
  }
  const std::string cmd = in.substr(s, e - s);
  *at = e;
  if (cmd == "left" || cmd == "right") return "";
  if (cmd == "cdot" || cmd == "times") return "*";
  if (cmd == "pi") return "pi";
  if (cmd == "theta" || cmd == "vartheta") return "theta";
  if (cmd == "phi" || cmd == "varphi") return "phi";
  if (cmd == "frac") {
    skip_spaces(in, at);
    const std::string num = take_group(in, at, '{', '}');
    skip_spaces(in, at);
    const std::string den = take_group(in, at, '{', '}');
    return "(" + to_infix(num) + ")/(" + to_infix(den) + ")";
  }
  if (cmd == "sqrt") {
    skip_spaces(in, at);
    return "sqrt(" + to_infix(take_group(in, at, '{', '}')) + ")";
  }
  std::string fn = cmd;
  if (cmd == "ln") fn = "log";
  else if (cmd == "arcsin") fn = "asin";
  else if (cmd == "arccos") fn = "acos";
  else if (cmd == "arctan") fn = "atan";
  else if (cmd == "operatorname") {
    skip_spaces(in, at);
    fn = lower(take_group(in, at, '{', '}'));
  }
  static const char* one[] = {"sin", "cos", "tan", "sinh", "cosh", "tanh", "asin", "acos", "atan", "exp",
                              "log", "abs", "floor", "ceil", "round", "sign", "sgn", "erf"};
  for (const char* f : one) {
    if (fn != f) continue;
    // argument: a {group}, a (group), a command, one letter or a number
    skip_spaces(in, at);
    if (*at >= in.size()) throw Failure{"missing function argument"};
    std::string arg;
    const char c = in[*at];
    if (c == '{') {
      arg = to_infix(take_group(in, at, '{', '}'));
    } else if (c == '(') {
      arg = to_infix(take_group(in, at, '(', ')'));
    } else if (c == '\\') {
      arg = command(in, at);
      if (arg.empty()) throw Failure{"invalid function argument"};
    } else if (is_alpha(c)) {
      arg = std::string(1, c);
      ++*at;
    } else if (std::isdigit(static_cast<unsigned char>(c)) || c == '.') {
      const char* p0 = in.c_str() + *at;
      char* p1 = nullptr;
      std::strtod(p0, &p1);
      if (p1 == p0) throw Failure{"invalid number in argument"};
      arg = in.substr(*at, (size_t)(p1 - p0));
      *at += (size_t)(p1 - p0);
    } else {
      throw Failure{"unsupported function argument"};
    }
    if (fn == "sgn") fn = "sign";
    return fn + "(" + arg + ")";
  }
  if (fn == "min" || fn == "max" || fn == "atan2" || fn == "pow") {
    skip_spaces(in, at);
    std::string g;
    if (*at < in.size() && in[*at] == '{')
      g = take_group(in, at, '{', '}');
    else if (*at < in.size() && in[*at] == '(')
      g = take_group(in, at, '(', ')');
    else
      throw Failure{"expected arguments for " + fn};
    int depth = 0;
    size_t comma = std::string::npos;
    for (size_t q = 0; q < g.size(); ++q) {
      if (g[q] == '{' || g[q] == '(') ++depth;
      else if (g[q] == '}' || g[q] == ')') --depth;
      else if (g[q] == ',' && depth == 0) {
        comma = q;
        break;
      }
    }
    if (comma == std::string::npos) throw Failure{fn + " requires two arguments separated by comma"};
    return fn + "(" + to_infix(g.substr(0, comma)) + "," + to_infix(g.substr(comma + 1)) + ")";
  }
  throw Failure{"unsupported latex command: \\" + cmd};
}

std::string to_infix(const std::string& in) {
  std::string out;
  size_t at = 0;
  while (at < in.size()) {
    const char c = in[at];
    if (is_space(c) || c == '$') {
      ++at;
    } else if (c == '\\') {
      out += command(in, &at);
    } else if (c == '{') {
      out += "(" + to_infix(take_group(in, &at, '{', '}')) + ")";
    } else if (c == '}') {
      throw Failure{"unexpected '}' in expression"};
    } else {
      out.push_back(c);
      ++at;
    }
  }
  return out;
}

struct Tok {
  enum Kind { Num, Id, Plus, Minus, Star, Slash, Caret, LP, RP, Comma, End } kind;
  double v;
  std::string s;
};

std::vector<Tok> tokenize(const std::string& s) {
  std::vector<Tok> out;
  size_t at = 0;
  while (at < s.size()) {
    const char c = s[at];
    if (is_space(c)) {
      ++at;
    } else if (std::isdigit(static_cast<unsigned char>(c)) || c == '.') {
      const char* p0 = s.c_str() + at;
      char* p1 = nullptr;
      const double v = std::strtod(p0, &p1);
      if (p1 == p0) throw Failure{"invalid number in expression"};
      out.push_back({Tok::Num, v, {}});
      at += (size_t)(p1 - p0);
    } else if (is_alpha(c)) {
      size_t e = at + 1;
      while (e < s.size() && is_alpha(s[e])) ++e;
      out.push_back({Tok::Id, 0.0, lower(s.substr(at, e - at))});
      at = e;
    } else {
      Tok::Kind k;
      switch (c) {
        case '+': k = Tok::Plus; break;
        case '-': k = Tok::Minus; break;
        case '*': k = Tok::Star; break;
        case '/': k = Tok::Slash; break;
        case '^': k = Tok::Caret; break;
        case '(': k = Tok::LP; break;
        case ')': k = Tok::RP; break;
        case ',': k = Tok::Comma; break;
        default: throw Failure{std::string("unexpected token: ") + c};
      }
      out.push_back({k, 0.0, {}});
      ++at;
    }
  }
  out.push_back({Tok::End, 0.0, {}});
  return out;
}

// Recursive descent with the reference's levels: sum > product (explicit or
// implicit) > power (right-associative, unary base) > unary > primary. Emits
// postfix code directly.
class Compiler {
 public:
  explicit Compiler(std::vector<Tok> t) : tk_(std::move(t)) {}

  void run(ExprProg* P) {
    prog_ = P;
    P->n = 0;
    sum();
    if (peek().kind != Tok::End) throw Failure{"unexpected trailing tokens"};
    // stack depth of the program
    int sp = 0, mx = 0;
    for (int q = 0; q < P->n; ++q) {
      const int op = P->op[q];
      if (op <= kT)
        ++sp;
      else if (op == kAdd || op == kSub || op == kMul || op == kDiv || op == kPow || op == kMin || op == kMax ||
               op == kAtan2 || op == kPow2)
        --sp;
      if (sp > mx) mx = sp;
    }
    if (mx > kExprMaxStack) throw Failure{"expression too large for the device evaluator"};
    P->depth = mx;
  }

 private:
  struct Depth {
    int& d;
    explicit Depth(int& x) : d(x) {
      if (++d > kExprMaxDepth)
        throw Failure{"expression too deeply nested (max depth: " + std::to_string(kExprMaxDepth) + ")"};
    }
    ~Depth() { --d; }
  };

  const Tok& peek() const { return tk_[at_]; }
  bool match(Tok::Kind k) {
    if (peek().kind != k) return false;
    if (at_ + 1 < tk_.size()) ++at_;
    return true;
  }
  void emit(int op, double v = 0.0) {
    if (prog_->n >= kExprMaxOps) throw Failure{"expression too large for the device evaluator"};
    prog_->op[prog_->n] = (uint8_t)op;
    prog_->val[prog_->n] = v;
    ++prog_->n;
  }

  void sum() {
    Depth g(depth_);
    product();
    while (true) {
      if (match(Tok::Plus)) {
        product();
        emit(kAdd);
      } else if (match(Tok::Minus)) {
        product();
        emit(kSub);
      } else {
        break;
      }
    }
  }
  void product() {
    Depth g(depth_);
    power();
    while (true) {
      if (match(Tok::Star)) {
        power();
        emit(kMul);
      } else if (match(Tok::Slash)) {
        power();
        emit(kDiv);
      } else if (peek().kind == Tok::Num || peek().kind == Tok::Id || peek().kind == Tok::LP) {
        power();
        emit(kMul);
      } else {
        break;
      }
    }
  }
  void power() {
    Depth g(depth_);
    unary();
    if (match(Tok::Caret)) {
      power();
      emit(kPow);
    }
  }
  void unary() {
    Depth g(depth_);
    if (match(Tok::Plus)) {
      unary();
      return;
    }
    if (match(Tok::Minus)) {
      unary();
      emit(kNeg);
      return;
    }
    primary();
  }
  void primary() {
    if (match(Tok::Num)) {
      emit(kNum, tk_[at_ - 1].v);
      return;
    }
    if (match(Tok::Id)) {
      const std::string name = tk_[at_ - 1].s;
      if (name == "x" || name == "r") return emit(kX);
      if (name == "y" || name == "theta") return emit(kY);
      if (name == "z" || name == "phi") return emit(kZ);
      if (name == "t") return emit(kT);
      if (name == "pi") return emit(kNum, kExprPi);
      if (name == "e") return emit(kNum, std::exp(1.0));
      if (!match(Tok::LP)) throw Failure{"unknown identifier: " + name};
      sum();
      bool two = false;
      if ((name == "min" || name == "max" || name == "atan2" || name == "pow") && match(Tok::Comma)) {
        sum();
        two = true;
      }
      if (!match(Tok::RP)) throw Failure{"missing closing parenthesis for function"};
      if (name == "min" || name == "max" || name == "atan2" || name == "pow") {
        if (!two) emit(kNum, 0.0);  // a missing second argument is 0
        emit(name == "min" ? kMin : name == "max" ? kMax : name == "atan2" ? kAtan2 : kPow2);
        return;
      }
      static const struct {
        const char* name;
        int op;
      } fns[] = {{"sin", kSin},     {"cos", kCos},   {"tan", kTan},   {"sinh", kSinh},   {"cosh", kCosh},
                 {"tanh", kTanh},   {"asin", kAsin}, {"acos", kAcos}, {"atan", kAtan},   {"exp", kExp},
                 {"log", kLog},     {"sqrt", kSqrt}, {"floor", kFloor}, {"ceil", kCeil}, {"round", kRound},
                 {"abs", kAbs},     {"sign", kSign}, {"erf", kErf}};
      for (const auto& f : fns)
        if (name == f.name) return emit(f.op);
      emit(kZero1);  // any other name evaluates its argument and gives 0
      return;
    }
    if (match(Tok::LP)) {
      sum();
      if (!match(Tok::RP)) throw Failure{"missing closing parenthesis"};
      return;
    }
    throw Failure{"unexpected token in expression"};
  }

  std::vector<Tok> tk_;
  size_t at_ = 0;
  int depth_ = 0;
  ExprProg* prog_ = nullptr;
};

void compile(const std::string& latex, ExprProg* P) {
  const std::string infix = to_infix(latex);
  if (infix.empty()) throw Failure{"empty expression"};
  Compiler c(tokenize(infix));
  c.run(P);
}

void copy_msg(char* dst, size_t len, const std::string& m) {
  if (!dst || len == 0) return;
  std::strncpy(dst, m.c_str(), len - 1);
  dst[len - 1] = '\0';
}

// Node map of the whole grid (face < 0) or of one face in the face-local
// order of pdeb200_face arrays: left/right j + ny*k, bottom/top i + nx*k,
// front/back i + nx*j. 2D grids have z = 0.
pdeb200_status grid_map(const pdeb200_problem* g, int face, NodeMap* m, long long* n) {
  const int nz = g->nz > 1 ? g->nz : 1;
  if (g->nx < 2 || g->ny < 2 || (face >= 4 && nz < 2)) return PDEB200_ERR_INVALID;
  const double dx = (g->xmax - g->xmin) / (g->nx - 1);
  const double dy = (g->ymax - g->ymin) / (g->ny - 1);
  const double dz = nz > 1 ? (g->zmax - g->zmin) / (nz - 1) : 0.0;
  const double lo[3] = {g->xmin, g->ymin, nz > 1 ? g->zmin : 0.0};
  const double hi[3] = {g->xmax, g->ymax, nz > 1 ? g->zmax : 0.0};
  const double h[3] = {dx, dy, dz};
  const int dims[3] = {g->nx, g->ny, nz};
  int fixed = face < 0 ? -1 : face / 2;  // axis held at a boundary value
  int idx = 0, sizes[3] = {1, 1, 1};
  for (int c = 0; c < 3; ++c) {
    m->base[c] = lo[c];
    m->step[c] = h[c];
    if (c == fixed) {
      m->axis[c] = 3;
      m->base[c] = (face & 1) ? hi[c] : lo[c];
    } else if (c == 2 && nz == 1) {
      m->axis[c] = 3;
      m->base[c] = 0.0;
    } else {
      m->axis[c] = idx;
      sizes[idx++] = dims[c];
    }
  }
  m->na = sizes[0];
  m->nb = sizes[1];
  *n = (long long)sizes[0] * sizes[1] * sizes[2];
  return PDEB200_OK;
}

pdeb200_status run_eval(const ExprProg* P, const NodeMap& m, long long n, double t, int device, double* out,
                        int mem_space, char* message, size_t message_len) {
  try {
    Context* ctx = get_context(device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    Buf prog(sizeof(ExprProg), ctx->stream);
    PDEB_CUDA(cudaMemcpyAsync(prog.as<void>(), P, sizeof(ExprProg), cudaMemcpyHostToDevice, ctx->stream));
    double* d_out = out;
    Buf ob;
    if (mem_space != PDEB200_MEM_DEVICE) {
      ob = Buf(sizeof(double) * n, ctx->stream);
      d_out = ob.as<double>();
    }
    const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)ctx->num_sms * 16);
    k_eval_expr<<<blocks, 256, 0, ctx->stream>>>(prog.as<ExprProg>(), m, n, t, d_out);
    PDEB_CUDA(cudaGetLastError());
    ctx->count();
    if (mem_space != PDEB200_MEM_DEVICE)
      PDEB_CUDA(cudaMemcpyAsync(out, d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
  } catch (const StatusFailure& s) {
    copy_msg(message, message_len, s.what);
    return s.status;
  } catch (const CudaFailure& c) {
    copy_msg(message, message_len, c.what);
    cudaGetLastError();
    return PDEB200_ERR_CUDA;
  }
  return PDEB200_OK;
}

}  // namespace
}  // namespace pdeb

extern "C" {

pdeb200_status pdeb200_expression_value(const char* latex, double x, double y, double z, double t, double* value,
                                        char* message, size_t message_len) {
  using namespace pdeb;
  copy_msg(message, message_len, "");
  if (!latex || !value) return PDEB200_ERR_INVALID;
  auto P = std::make_unique<ExprProg>();
  try {
    compile(latex, P.get());
  } catch (const Failure& f) {
    copy_msg(message, message_len, f.what);
    return PDEB200_ERR_INVALID;
  }
  *value = expr_run(*P, x, y, z, t);
  return PDEB200_OK;
}

pdeb200_status pdeb200_eval_expression(const char* latex, const pdeb200_problem* grid, double t, int32_t device,
                                       double* out, int32_t mem_space, char* message, size_t message_len) {
  using namespace pdeb;
  copy_msg(message, message_len, "");
  if (!latex || !grid || !out) return PDEB200_ERR_INVALID;
  auto P = std::make_unique<ExprProg>();
  try {
    compile(latex, P.get());
  } catch (const Failure& f) {
    copy_msg(message, message_len, f.what);
    return PDEB200_ERR_INVALID;
  }
  NodeMap m{};
  long long n = 0;
  pdeb200_status st = grid_map(grid, -1, &m, &n);
  if (st != PDEB200_OK) {
    copy_msg(message, message_len, "grid must have at least 2 nodes per dimension");
    return st;
  }
  m.has_prog = 1;
  return run_eval(P.get(), m, n, t, device, out, mem_space, message, message_len);
}

pdeb200_status pdeb200_eval_face_expression(const char* latex, const double* linear, const pdeb200_problem* grid,
                                            int32_t face, double t, int32_t device, double* out, int32_t mem_space,
                                            char* message, size_t message_len) {
  using namespace pdeb;
  copy_msg(message, message_len, "");
  if (!grid || !out || face < 0 || face > 5) return PDEB200_ERR_INVALID;
  auto P = std::make_unique<ExprProg>();
  P->n = 0;
  bool parsed = false;
  if (latex && latex[0]) {
    try {
      compile(latex, P.get());
      parsed = true;
    } catch (const Failure&) {
      P->n = 0;  // an expression that does not parse leaves the linear form
    }
  }
  NodeMap m{};
  long long n = 0;
  pdeb200_status st = grid_map(grid, face, &m, &n);
  if (st != PDEB200_OK) {
    copy_msg(message, message_len, "grid must have at least 2 nodes per dimension (3D faces need nz > 1)");
    return st;
  }
  m.has_prog = parsed ? 1 : 0;
  m.linear = 1;
  for (int q = 0; q < 4; ++q) m.lin[q] = linear ? linear[q] : 0.0;
  return run_eval(P.get(), m, n, t, device, out, mem_space, message, message_len);
}

}  // extern "C"
