// Circuit front ends: OpenQASM 2 as written by qiskit / cirq, timed qasm,
// ProjectQ's command log and Quil (qasm_parser.c:12-1098).  Each reader
// fills a circuit with one gate per instruction line and reports the number
// of qubits, like the reference:
//   qiskit_qasm_read   gates at times 1, 2, 3, ... in file order, qubit q of
//                      the file becomes N - 1 - q (qiskit's ordering,
//                      qasm_parser.c:808-820); barriers take a time slot
//                      but add no gate
//   cirq_qasm_read     the same with the file's qubit numbers kept
//   qiskit_tqasm_read  "gate qr[i] @t;": the time is the @ field
//   projectq_qasm_read "Allocate | Qureg[i]" lines count the qubits, then
//                      "H | Qureg[0]", "CX | ( Qureg[0], Qureg[1] )",
//                      "Rz(0.5) | Qureg[1]" ... at times 1, 2, ... until
//                      "Deallocate"
//   quil_read          "H 0", "CNOT 0 1", "RX(pi/2) 3", PRAGMA lines
//                      skipped, times 1, 2, ...; the qubit count is one
//                      more than the largest qubit named
// Angles are arithmetic expressions in numbers and pi (+ - * / and
// parentheses), which covers every form the reference accepts (pi*x,
// x*pi/y, pi/x, x*pi, -pi/2, plain numbers; qasm_parser.c:521-575).
// Where the reference's own parsing is wrong for a well-formed line (Quil
// angles such as 3*pi/4, which its digit scan turns into pi/4, and a
// two-qubit Quil gate whose second qubit is 0, qasm_parser.c:74-112,
// 181-188), these readers take the line's meaning.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "runtime.h"

namespace quac {
namespace {

struct Expr {
  const char *p;
  bool ok = true;
  void ws() { while (*p && isspace((unsigned char)*p)) p++; }
  double prim() {
    ws();
    if (*p == '(') {
      p++;
      double v = sum();
      ws();
      if (*p == ')') p++; else ok = false;
      return v;
    }
    if (*p == '-') { p++; return -prim(); }
    if (*p == '+') { p++; return prim(); }
    if (strncmp(p, "pi", 2) == 0) { p += 2; return M_PI; }
    char *end = nullptr;
    const double v = strtod(p, &end);
    if (end == p) { ok = false; return 0.0; }
    p = end;
    return v;
  }
  double prod() {
    double v = prim();
    for (;;) {
      ws();
      if (*p == '*') { p++; v *= prim(); }
      else if (*p == '/') { p++; v /= prim(); }
      else return v;
    }
  }
  double sum() {
    double v = prod();
    for (;;) {
      ws();
      if (*p == '+') { p++; v += prod(); }
      else if (*p == '-') { p++; v -= prod(); }
      else return v;
    }
  }
};

bool eval_angle(const std::string &s, double &v) {
  Expr e{s.c_str()};
  v = e.sum();
  e.ws();
  return e.ok && *e.p == 0;
}

// "name(a,b,c)" -> name, {a, b, c}
void split_call(const std::string &tok, std::string &name, std::vector<std::string> &args) {
  const size_t lp = tok.find('(');
  args.clear();
  if (lp == std::string::npos) { name = tok; return; }
  name = tok.substr(0, lp);
  const size_t rp = tok.rfind(')');
  std::string inner = tok.substr(lp + 1, rp == std::string::npos ? std::string::npos : rp - lp - 1);
  int depth = 0;
  std::string cur;
  for (char ch : inner) {
    if (ch == '(') depth++;
    if (ch == ')') depth--;
    if (ch == ',' && depth == 0) { args.push_back(cur); cur.clear(); }
    else cur += ch;
  }
  args.push_back(cur);
}

std::string lower(std::string s) {
  for (auto &c : s) c = (char)tolower((unsigned char)c);
  return s;
}

std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) a++;
  while (b > a && isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

struct Gate {
  int type;
  std::vector<int> q;
  double th = 0, ph = 0, la = 0;
  double time = 0;
};

bool read_lines(const char *fn, std::vector<std::string> &lines, const char *who) {
  std::ifstream f(fn);
  if (!f) { fail(1, "ERROR! File not found in %s!\n", who); return false; }
  std::string l;
  while (std::getline(f, l)) lines.push_back(l);
  return true;
}

// the circuit, one gate per entry; quac_add_gate checks each gate's qubit count
void emit(circuit *circ, const std::vector<Gate> &gates) {
  create_circuit(circ, (PetscInt)gates.size());
  for (const Gate &g : gates)
    if (quac_add_gate(circ, g.time, g.type, (int)g.q.size(), g.q.data(), g.th, g.ph, g.la, nullptr, nullptr))
      return;
}

// qasm gate (qiskit names) with its angle list; false for an unknown name
bool qasm_gate(const std::string &name, const std::vector<std::string> &args, Gate &g) {
  double a[3] = {0, 0, 0};
  for (size_t k = 0; k < args.size() && k < 3; k++)
    if (!eval_angle(args[k], a[k])) return false;
  const std::string n = lower(name);
  if (n == "cx") g.type = CNOT;
  else if (n == "cz") g.type = CZ;
  else if (n == "h") g.type = HADAMARD;
  else if (n == "x") g.type = SIGMAX;
  else if (n == "y") g.type = SIGMAY;
  else if (n == "z") g.type = SIGMAZ;
  else if (n == "id") g.type = EYE;
  else if (n == "rx") { g.type = RX; g.th = a[0]; }
  else if (n == "ry") { g.type = RY; g.th = a[0]; }
  else if (n == "rz") { g.type = RZ; g.th = a[0]; }
  else if (n == "u1") { g.type = U1; g.la = a[0]; }                      // u1(l) = u3(0, 0, l)
  else if (n == "u2") { g.type = U2; g.th = M_PI / 2; g.ph = a[0]; g.la = a[1]; }  // u2(p, l) = u3(pi/2, p, l)
  else if (n == "u3") { g.type = U3; g.th = a[0]; g.ph = a[1]; g.la = a[2]; }
  else return false;
  return true;
}

// operands "qr[1],qr[2]" (any register name) -> qubit numbers
bool qasm_operands(const std::string &s, std::vector<int> &q) {
  q.clear();
  size_t i = 0;
  while ((i = s.find('[', i)) != std::string::npos) {
    const size_t j = s.find(']', i);
    if (j == std::string::npos) return false;
    q.push_back(atoi(s.substr(i + 1, j - i - 1).c_str()));
    i = j + 1;
  }
  return !q.empty();
}

int qasm_read(const char *fn, PetscInt *nq, circuit *circ, bool reverse, bool timed, const char *who) {
  std::vector<std::string> lines;
  if (!read_lines(fn, lines, who)) return 1;
  std::vector<Gate> gates;
  bool found = false;
  double time = 1.0;
  *nq = 0;
  for (const std::string &raw : lines) {
    std::string l = raw;
    const size_t cm = l.find("//");
    if (cm != std::string::npos) l = l.substr(0, cm);
    l = trim(l);
    if (l.empty()) continue;
    if (!found) {
      if (l.rfind("qreg", 0) == 0) {
        std::vector<int> q;
        if (!qasm_operands(l, q)) { fail(0, "ERROR! could not read the qreg line in %s\n", who); return 1; }
        *nq = q[0];
        found = true;
      }
      continue;  // header (OPENQASM, include)
    }
    if (l.rfind("creg", 0) == 0 || l.rfind("measure", 0) == 0) continue;
    // instruction: name[(args)] operands [@time];
    size_t sp = 0;
    int depth = 0;
    for (; sp < l.size(); sp++) {
      if (l[sp] == '(') depth++;
      if (l[sp] == ')') depth--;
      if (depth == 0 && isspace((unsigned char)l[sp])) break;
    }
    const std::string head = l.substr(0, sp);
    std::string rest = trim(l.substr(sp));
    double gtime = time;
    if (timed) {
      const size_t at = rest.find('@');
      if (at == std::string::npos) { fail(0, "ERROR! timed qasm line without @time: %s\n", raw.c_str()); return 1; }
      gtime = atof(rest.c_str() + at + 1);
      rest = rest.substr(0, at);
    }
    if (lower(head).rfind("barrier", 0) == 0) {
      if (!timed) time += 1.0;
      continue;
    }
    std::string name;
    std::vector<std::string> args;
    split_call(head, name, args);
    Gate g;
    if (!qasm_gate(name, args, g)) {
      fail(0, "%s\nERROR! Gate type not recognized in %s!\n", head.c_str(), who);
      return 1;
    }
    if (!qasm_operands(rest, g.q)) {
      fail(0, "ERROR! could not read the qubits of: %s\n", raw.c_str());
      return 1;
    }
    if (reverse)
      for (int &q : g.q) q = (int)*nq - q - 1;
    g.time = gtime;
    gates.push_back(g);
    if (!timed) time += 1.0;
  }
  if (!found) { fail(0, "ERROR! no qreg line in %s\n", who); return 1; }
  emit(circ, gates);
  return has_error() ? 1 : 0;
}

}  // namespace
}  // namespace quac

using namespace quac;

extern "C" {

void qiskit_qasm_read(char filename[], PetscInt *num_qubits, circuit *circ) {
  qasm_read(filename, num_qubits, circ, true, false, "qiskit_qasm_read");
}

void cirq_qasm_read(char filename[], PetscInt *num_qubits, circuit *circ) {
  qasm_read(filename, num_qubits, circ, false, false, "cirq_qasm_read");
}

void qiskit_tqasm_read(char filename[], PetscInt *num_qubits, circuit *circ) {
  qasm_read(filename, num_qubits, circ, false, true, "qiskit_tqasm_read");
}

void projectq_qasm_read(char filename[], PetscInt *num_qubits, circuit *circ) {
  std::vector<std::string> lines;
  if (!read_lines(filename, lines, "projectq_qasm_read")) return;
  std::vector<Gate> gates;
  double time = 1.0;
  *num_qubits = 0;
  bool allocating = true;
  for (const std::string &raw : lines) {
    std::string l;
    for (char ch : raw)
      if (!isspace((unsigned char)ch)) l += ch;  // whitespace removed, as the reference does
    if (l.empty()) continue;
    if (allocating && l.find("Allocate") != std::string::npos && l.find("Deallocate") == std::string::npos) {
      (*num_qubits)++;
      continue;
    }
    allocating = false;
    if (l.find("Deallocate") != std::string::npos) break;
    const size_t bar = l.find('|');
    if (bar == std::string::npos) continue;
    std::string name;
    std::vector<std::string> args;
    split_call(l.substr(0, bar), name, args);
    Gate g;
    double a = 0.0;
    if (!args.empty() && !eval_angle(args[0], a)) { fail(0, "ERROR! bad angle in: %s\n", raw.c_str()); return; }
    if (name == "CX") g.type = CNOT;
    else if (name == "H") g.type = HADAMARD;
    else if (name == "X") g.type = SIGMAX;
    else if (name == "Y") g.type = SIGMAY;
    else if (name == "Z") g.type = SIGMAZ;
    else if (name == "Rx") { g.type = RX; g.th = a; }
    else if (name == "Ry") { g.type = RY; g.th = a; }
    else if (name == "Rz") { g.type = RZ; g.th = a; }
    else { fail(0, "%s\nERROR! Gate type not recognized in projectq_qasm_read!\n", name.c_str()); return; }
    std::string ops = l.substr(bar + 1);
    for (auto &c : ops)
      if (c == '(' || c == ')') c = ' ';
    size_t i = 0;
    while ((i = ops.find("Qureg[", i)) != std::string::npos) {
      g.q.push_back(atoi(ops.c_str() + i + 6));
      i += 6;
    }
    g.time = time;
    time += 1.0;
    gates.push_back(g);
  }
  emit(circ, gates);
}

void quil_read(char filename[], PetscInt *num_qubits, circuit *circ) {
  std::vector<std::string> lines;
  if (!read_lines(filename, lines, "quil_read")) return;
  std::vector<Gate> gates;
  double time = 1.0;
  int maxq = -1;
  for (const std::string &raw : lines) {
    const std::string l = trim(raw);
    if (l.empty() || l.find("PRAGMA") != std::string::npos) continue;
    std::istringstream in(l);
    std::string head, tok;
    in >> head;
    std::string name;
    std::vector<std::string> args;
    split_call(head, name, args);
    Gate g;
    double a = 0.0;
    if (!args.empty() && !eval_angle(args[0], a)) { fail(0, "ERROR! bad angle in: %s\n", raw.c_str()); return; }
    if (name == "CNOT") g.type = CNOT;
    else if (name == "CZ") g.type = CZ;
    else if (name == "I") g.type = EYE;
    else if (name == "H") g.type = HADAMARD;
    else if (name == "X") g.type = SIGMAX;
    else if (name == "Y") g.type = SIGMAY;
    else if (name == "Z") g.type = SIGMAZ;
    else if (name == "RX") { g.type = RX; g.th = a; }
    else if (name == "RY") { g.type = RY; g.th = a; }
    else if (name == "RZ") { g.type = RZ; g.th = a; }
    else { fail(0, "%s\nERROR! Gate type not recognized in quil_read!\n", name.c_str()); return; }
    while (in >> tok) {
      g.q.push_back(atoi(tok.c_str()));
      maxq = std::max(maxq, g.q.back());
    }
    g.time = time;
    time += 1.0;
    gates.push_back(g);
  }
  *num_qubits = maxq + 1;
  emit(circ, gates);
}

}  // extern "C"
