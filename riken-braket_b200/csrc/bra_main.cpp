// rbk-bra: command-line drop-in for bra's nompi executable (bra/src/bra.cpp:63-110,
// :290-330) running .qcx programs on the B200 engine.
//
//   rbk-bra [--file <path>] [--seed <seed>] [--threads <n>] [--precision c128|c64]
//           [--device <id>] [--unfused] [--no-timing]
//
// Without --file the program is read from standard input, as bra does.
// --threads is accepted for compatibility and has no effect.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

#include "rbk_qcx.h"

namespace {

void usage(std::ostream& o)
{
  o << "usage: rbk-bra [--file <path>] [--seed <seed>] [--threads <n>] [--precision c128|c64]\n"
       "               [--device <id>] [--unfused] [--no-timing]\n";
}

}  // namespace

int main(int argc, char** argv)
{
  rbk_qcx_options opt;
  rbk_qcx_default_options(&opt);
  std::string file;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto value = [&]() -> std::string {
      if (i + 1 >= argc) {
        std::cerr << "Error: " << a << " needs a value\n";
        usage(std::cerr);
        std::exit(EXIT_FAILURE);
      }
      return argv[++i];
    };
    if (a == "-h" || a == "--help") {
      usage(std::cout);
      return EXIT_SUCCESS;
    } else if (a == "-f" || a == "--file") {
      file = value();
    } else if (a == "--seed") {
      opt.seed = std::strtoull(value().c_str(), nullptr, 10);
    } else if (a == "--threads") {
      value();
    } else if (a == "--precision") {
      const std::string p = value();
      if (p == "c128" || p == "double") opt.precision = RBK_C128;
      else if (p == "c64" || p == "float") opt.precision = RBK_C64;
      else {
        std::cerr << "Error: unknown precision " << p << "\n";
        return EXIT_FAILURE;
      }
    } else if (a == "--device") {
      opt.device = std::atoi(value().c_str());
    } else if (a == "--unfused") {
      opt.deferred = 0;
    } else if (a == "--no-timing") {
      opt.print_timing = 0;
    } else {
      std::cerr << "Error: unknown option " << a << "\n";
      usage(std::cerr);
      return EXIT_FAILURE;
    }
  }
  std::stringstream buf;
  if (file.empty()) {
    buf << std::cin.rdbuf();
  } else {
    std::ifstream in(file);
    if (!in) {
      std::cerr << "Error: cannot open " << file << "\n";
      return EXIT_FAILURE;
    }
    buf << in.rdbuf();
  }
  const std::string text = buf.str();
  rbk_qcx_program* prog = nullptr;
  if (rbk_qcx_parse(text.data(), text.size(), &prog) != RBK_OK) {
    std::cerr << "Error: " << rbk_last_error() << "\n";
    return EXIT_FAILURE;
  }
  char* out = nullptr;
  const int rc = rbk_qcx_run(prog, &opt, &out, nullptr);
  rbk_qcx_destroy(prog);
  if (rc != RBK_OK) {
    std::cerr << "Error: " << rbk_last_error() << "\n";
    return EXIT_FAILURE;
  }
  std::fputs(out, stdout);
  std::fflush(stdout);
  rbk_qcx_free_text(out);
  return EXIT_SUCCESS;
}
