// hvm64 -- command line front end of the B200 reducer (the reference's
// `hvm64 run` / `hvm64 reduce` / `hvm64 transform`, src/main.rs:32-204 and
// src/args.rs), calling only the C ABI in hvm64.h.
//
//   hvm64 run FILE [ARGS..] [-e ENTRY] [-m MEM] [-s] [TRANSFORM OPTS]
//   hvm64 reduce [FILES..] [-m MEM] [-s] [TRANSFORM OPTS] -- EXPRS..
//   hvm64 transform [FILES..] [TRANSFORM OPTS]
//
// `run` boots ENTRY (default main) applied to each ARG in turn
// (apply_tree, src/main.rs:195-204); `reduce` normalises each expression
// against the Book of FILES.  Each normal form goes to stdout; with -s the
// Rewrites block and TIME / RPS go to stderr as the reference prints them.
// --print-net prints the net that would be reduced instead of reducing it.
// `transform` prints the Book after its passes (src/main.rs:71-74).
// TRANSFORM OPTS (src/args.rs:43-133): -O PASSES (pre-reduce | pre, all, and
// their no- forms; the Book passes eta-reduce, inline and prune are not part
// of this build), --pre-reduce-skip NAMES, --pre-reduce-memory MEM,
// --pre-reduce-rewrites N (default 100M).  `run` never pre-reduces its entry
// (src/main.rs:58-61).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "hvm64.h"

namespace {

void usage() {
  fprintf(stderr,
          "usage: hvm64 run FILE [ARGS..] [-e ENTRY] [-m MEM] [-s] [-O PASSES]\n"
          "       hvm64 reduce [FILES..] [-m MEM] [-s] [-O PASSES] -- EXPRS..\n"
          "       hvm64 transform [FILES..] [-O PASSES] [--pre-reduce-skip NAMES]\n"
          "                       [--pre-reduce-memory MEM] [--pre-reduce-rewrites N]\n");
}

// -O values (src/args.rs:128-133 and the `all` switch): the pass flags in
// the order given, the last word winning.  Returns false on an unknown name.
struct Passes {
  bool pre_reduce = false, eta = false, inline_ = false, prune = false;
};
bool apply_pass(const std::string& word, Passes* p) {
  bool on = true;
  std::string w = word;
  if (w.rfind("no-", 0) == 0) {
    on = false;
    w = w.substr(3);
  }
  if (w == "all") *p = Passes{on, on, on, on};
  else if (w == "pre-reduce" || w == "pre") p->pre_reduce = on;
  else if (w == "eta-reduce" || w == "eta") p->eta = on;
  else if (w == "inline") p->inline_ = on;
  else if (w == "prune") p->prune = on;
  else return false;
  return true;
}

// util/src/parse_abbrev_number.rs: a number with an optional K/M/G/T suffix.
bool parse_mem(const std::string& s, unsigned long long* out) {
  if (s.empty()) return false;
  unsigned long long scale = 1;
  std::string digits = s;
  char last = s.back();
  const char* suf = "KMGT";
  for (int i = 0; i < 4; i++)
    if (last == suf[i] || last == suf[i] + 32) {
      scale = 1ull << (10 * (i + 1));
      digits = s.substr(0, s.size() - 1);
    }
  char* end = nullptr;
  unsigned long long v = strtoull(digits.c_str(), &end, 10);
  if (digits.empty() || *end) return false;
  *out = v * scale;
  return true;
}

bool read_file(const std::string& path, std::string* out) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  char buf[1 << 16];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) out->append(buf, n);
  fclose(f);
  return true;
}

// The net `run` reduces: ENTRY applied to each argument in turn.  Each
// application rebinds the root r(k) to a fresh variable r(k+1) and adds the
// redex (arg r(k+1)) ~ r(k), as apply_tree does.
std::string run_net(const std::string& entry, const std::vector<std::string>& args) {
  std::string root = "@" + entry, redexes;
  for (size_t k = 0; k < args.size(); k++) {
    std::string v = "__hvm64_root" + std::to_string(k);
    redexes += " & (" + args[k] + " " + v + ") ~ " + root;
    root = v;
  }
  return root + redexes;
}

// src/main.rs:181-193: the statistics block, TIME and RPS.
void print_stats(const hvm64_rewrites& rw, double ms) {
  auto pretty = [](unsigned long long n) {
    std::string s = std::to_string(n), o;
    int head = int(s.size() % 3);
    for (size_t i = 0; i < s.size(); i++) {
      if (i && (int(i) - head) % 3 == 0) o += '_';
      o += s[i];
    }
    return o;
  };
  unsigned long long total = rw.anni + rw.comm + rw.eras + rw.dref + rw.oper;
  const char* names[] = {"RWTS   ", "- ANNI ", "- COMM ", "- ERAS ", "- DREF ", "- OPER "};
  unsigned long long vals[] = {total, rw.anni, rw.comm, rw.eras, rw.dref, rw.oper};
  for (int i = 0; i < 6; i++) fprintf(stderr, "%s: %15s\n", names[i], pretty(vals[i]).c_str());
  // TIME: a Duration's `{:.3?}`, i.e. in the largest unit whose whole part is
  // nonzero (s, ms, µs, ns), three decimals.
  double ns = ms * 1e6;
  if (ns >= 1e9) fprintf(stderr, "TIME   : %.3fs\n", ns / 1e9);
  else if (ns >= 1e6) fprintf(stderr, "TIME   : %.3fms\n", ns / 1e6);
  else if (ns >= 1e3) fprintf(stderr, "TIME   : %.3f\xc2\xb5s\n", ns / 1e3);
  else fprintf(stderr, "TIME   : %.3fns\n", ns);
  // RPS: total / whole milliseconds / 1000 as an f64 (inf or NaN under 1 ms)
  double whole_ms = floor(ms);
  double rps = whole_ms > 0 ? double(total) / whole_ms / 1000.0 : (total ? INFINITY : NAN);
  if (std::isinf(rps)) fprintf(stderr, "RPS    : inf M\n");
  else if (std::isnan(rps)) fprintf(stderr, "RPS    : NaN M\n");
  else fprintf(stderr, "RPS    : %.3f M\n", rps);
}

int fail(const char* what) {
  fprintf(stderr, "error: %s: %s\n", what, hvm64_last_error());
  return 101;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    usage();
    return 2;
  }
  std::string mode = argv[1];
  if (mode != "run" && mode != "reduce" && mode != "transform") {
    usage();
    return 2;
  }
  std::vector<std::string> files, args, exprs;
  std::string entry = "main", skip;
  unsigned long long mem = 0, pre_mem = 0, pre_rwts = 100ull << 20;
  bool stats = false, after_dd = false, print_only = false;
  Passes passes;
  for (int k = 2; k < argc; k++) {
    std::string a = argv[k];
    if (after_dd) {
      exprs.push_back(a);
    } else if (a == "--") {
      after_dd = true;
    } else if (a.rfind("-O", 0) == 0) {
      std::string v = a.size() > 2 ? a.substr(2) : (k + 1 < argc ? std::string(argv[++k]) : std::string());
      size_t s0 = 0;
      while (s0 <= v.size()) {  // value_delimiter ' '
        size_t e = v.find(' ', s0);
        if (e == std::string::npos) e = v.size();
        if (e > s0 && !apply_pass(v.substr(s0, e - s0), &passes)) {
          fprintf(stderr, "error: unknown transform pass %s\n", v.substr(s0, e - s0).c_str());
          return 2;
        }
        s0 = e + 1;
      }
    } else if (a == "--pre-reduce-skip" && k + 1 < argc) {
      skip += std::string(argv[++k]) + " ";
    } else if (a == "--pre-reduce-memory" && k + 1 < argc) {
      if (!parse_mem(argv[++k], &pre_mem)) {
        fprintf(stderr, "error: bad memory size %s\n", argv[k]);
        return 2;
      }
    } else if (a == "--pre-reduce-rewrites" && k + 1 < argc) {
      if (!parse_mem(argv[++k], &pre_rwts)) {
        fprintf(stderr, "error: bad rewrite count %s\n", argv[k]);
        return 2;
      }
    } else if (a == "-s" || a == "--stats") {
      stats = true;
    } else if (a == "--print-net") {
      print_only = true;
    } else if (a == "-1" || a == "--single") {
      // the reference's single-thread switch; the device reducer has one mode
    } else if ((a == "-m" || a == "--memory") && k + 1 < argc) {
      if (!parse_mem(argv[++k], &mem)) {
        fprintf(stderr, "error: bad memory size %s\n", argv[k]);
        return 2;
      }
    } else if (a == "-e" && k + 1 < argc) {
      entry = argv[++k];
    } else if (mode == "run" && files.empty()) {
      files.push_back(a);
    } else if (mode == "run") {
      args.push_back(a);
    } else {
      files.push_back(a);
    }
  }
  if (mode == "run" && files.empty()) {
    usage();
    return 2;
  }
  std::string text;
  for (auto& f : files) {
    if (!read_file(f, &text)) {
      fprintf(stderr, "Input file \"%s\" not found\n", f.c_str());
      return 1;
    }
    text += "\n";
  }
  if (passes.eta || passes.inline_ || passes.prune) {
    fprintf(stderr, "error: only the pre-reduce transform is part of this build\n");
    return 2;
  }
  if (passes.pre_reduce) {  // Book::transform (transform/src/transform.rs:35-77)
    if (mode == "run") skip += entry;
    size_t len = 0, nlen = 0;
    std::string out(4 * text.size() + 4096, '\0'), nn(4096, '\0');
    for (int pass = 0; pass < 2; pass++) {
      if (hvm64_pre_reduce(text.data(), text.size(), skip.c_str(), pre_rwts, pre_mem, nullptr, nullptr, &out[0],
                           out.size(), &len, &nn[0], nn.size(), &nlen))
        return fail("pre-reducing");
      if (len < out.size() && nlen < nn.size()) break;
      out.assign(len + 1, '\0');  // the Book outgrew the buffer: size it and run again
      nn.assign(nlen + 1, '\0');
    }
    out.resize(len);
    text = out + "\n";
  }
  if (mode == "transform") {  // src/main.rs:71-74: println!("{}", book)
    if (!passes.pre_reduce) {
      size_t len = 0;
      if (hvm64_book_format(text.data(), text.size(), nullptr, 0, &len)) return fail("parsing the book");
      std::string out(len + 1, '\0');
      hvm64_book_format(text.data(), text.size(), &out[0], out.size(), &len);
      out.resize(len);
      text = out + "\n";
    }
    printf("%s", text.c_str());
    return 0;
  }
  std::vector<std::string> nets;
  if (mode == "run") nets.push_back(run_net(entry, args));
  else nets = exprs;
  if (print_only) {
    for (auto& n : nets) printf("%s\n", n.c_str());
    return 0;
  }
  hvm64_book* book = nullptr;
  if (hvm64_book_load(text.data(), text.size(), &book)) return fail("loading the book");
  int rc = 0;
  for (auto& n : nets) {
    hvm64_net* net = nullptr;
    if (hvm64_net_create(book, mem, &net)) {
      rc = fail("creating the net");
      break;
    }
    hvm64_rewrites rw{};
    double ms = 0;
    if (hvm64_net_encode(net, n.data(), n.size()) || hvm64_net_normal(net, nullptr, &rw, &ms)) {
      rc = fail("reducing");
      hvm64_net_free(net);
      break;
    }
    size_t len = 0;
    hvm64_net_readback(net, nullptr, 0, &len);
    std::string out(len + 1, '\0');
    if (hvm64_net_readback(net, &out[0], out.size(), &len)) {
      rc = fail("reading back");
      hvm64_net_free(net);
      break;
    }
    out.resize(len);
    printf("%s\n", out.c_str());
    fflush(stdout);
    if (stats) print_stats(rw, ms);
    hvm64_net_free(net);
  }
  hvm64_book_free(book);
  return rc;
}
