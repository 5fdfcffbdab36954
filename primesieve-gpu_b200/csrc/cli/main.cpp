// primesieve CLI, counting subset, on the B200 engine.
//
//   primesieve [START] STOP [OPTION]...
//
// Drop-in for the reference's `primesieve ... --count[=NUM+] --gpu` path
// (src/app/main.cpp:132-254, option parsing src/app/CmdOptions.cpp:324-401,
// help src/app/help.cpp). Same option spellings, same output lines
// ("Primes: N", "Twin primes: N", ...; a bare number with -q and a single
// count; "Seconds: x.xxx" with --time, which is the default without -q).
// Also --nth-prime (main.cpp:256-290) and --print for primes (the primes
// extracted on the GPU). Differences: everything runs on the GPU, all
// requested counts come from one sieve pass; printing k-tuplets, RiemannR
// and the stress test of the reference are not part of this tool.
#include "../../../include/primesieve.hpp"
#include "../../../include/primesieve/gpu.hpp"
#include "calculator.hpp"

#include <array>
#include <chrono>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <map>
#include <string>
#include <vector>

namespace {

enum OptionId {
  OPT_COUNT, OPT_DIST, OPT_GPU, OPT_GPU_DEVICE, OPT_GPU_INFO, OPT_HELP,
  OPT_NUMBER, OPT_QUIET, OPT_SIZE, OPT_THREADS, OPT_TIME, OPT_VERSION,
  OPT_NO_STATUS, OPT_NTH_PRIME, OPT_PRINT, OPT_UNSUPPORTED
};
enum Param { NO_PARAM, REQUIRED_PARAM, OPTIONAL_PARAM };

struct Options {
  std::vector<uint64_t> numbers;
  int flags = 0;            // bit i: count kind i
  bool gpu = false;
  int gpu_device = -1;
  bool gpu_info = false;
  bool quiet = false;
  bool time = false;
  bool help = false;
  bool version = false;
  bool nth_prime = false;
  bool print = false;
};

struct Parsed { std::string str, opt, val; };

bool is_option(const std::string& s) {
  if (s.size() >= 2 && s[0] == '-' && std::isalpha((unsigned char) s[1])) return true;
  if (s.size() >= 3 && s[0] == '-' && s[1] == '-' && std::isalpha((unsigned char) s[2])) return true;
  return false;
}

const std::map<std::string, std::pair<OptionId, Param>>& option_map() {
  static const std::map<std::string, std::pair<OptionId, Param>> m = {
    { "-c", { OPT_COUNT, OPTIONAL_PARAM } }, { "--count", { OPT_COUNT, OPTIONAL_PARAM } },
    { "-d", { OPT_DIST, REQUIRED_PARAM } }, { "--dist", { OPT_DIST, REQUIRED_PARAM } },
    { "-g", { OPT_GPU, NO_PARAM } }, { "--gpu", { OPT_GPU, NO_PARAM } },
    { "--gpu-device", { OPT_GPU_DEVICE, REQUIRED_PARAM } },
    { "--gpu-info", { OPT_GPU_INFO, NO_PARAM } },
    { "-h", { OPT_HELP, NO_PARAM } }, { "--help", { OPT_HELP, NO_PARAM } },
    { "--number", { OPT_NUMBER, REQUIRED_PARAM } },
    { "-q", { OPT_QUIET, NO_PARAM } }, { "--quiet", { OPT_QUIET, NO_PARAM } },
    { "-s", { OPT_SIZE, REQUIRED_PARAM } }, { "--size", { OPT_SIZE, REQUIRED_PARAM } },
    { "-t", { OPT_THREADS, REQUIRED_PARAM } }, { "--threads", { OPT_THREADS, REQUIRED_PARAM } },
    { "--time", { OPT_TIME, NO_PARAM } },
    { "-v", { OPT_VERSION, NO_PARAM } }, { "--version", { OPT_VERSION, NO_PARAM } },
    { "--no-status", { OPT_NO_STATUS, NO_PARAM } },
    // reference modes outside the counting path
    { "-p", { OPT_PRINT, OPTIONAL_PARAM } }, { "--print", { OPT_PRINT, OPTIONAL_PARAM } },
    { "-n", { OPT_NTH_PRIME, NO_PARAM } }, { "--nth-prime", { OPT_NTH_PRIME, NO_PARAM } },
    { "--nthprime", { OPT_NTH_PRIME, NO_PARAM } },
    { "-R", { OPT_UNSUPPORTED, NO_PARAM } }, { "--RiemannR", { OPT_UNSUPPORTED, NO_PARAM } },
    { "--RiemannR-inverse", { OPT_UNSUPPORTED, NO_PARAM } },
    { "-S", { OPT_UNSUPPORTED, OPTIONAL_PARAM } }, { "--stress-test", { OPT_UNSUPPORTED, OPTIONAL_PARAM } },
    { "--test", { OPT_UNSUPPORTED, NO_PARAM } }, { "--cpu-info", { OPT_UNSUPPORTED, NO_PARAM } },
    { "--timeout", { OPT_UNSUPPORTED, REQUIRED_PARAM } },
  };
  return m;
}

[[noreturn]] void fail(const std::string& msg) { throw primesieve::primesieve_error(msg); }

// One command-line token (or token + value), reference CmdOptions.cpp:83-189.
Parsed parse_one(int argc, char** argv, int& i) {
  const auto& m = option_map();
  Parsed o;
  o.str = argv[i];
  if (o.str.empty()) fail("unrecognized option ''");
  auto it = m.find(o.str);
  if (it != m.end()) {
    o.opt = o.str;
    if (it->second.second == REQUIRED_PARAM) {
      i++;
      if (i < argc) o.val = argv[i];
      if (o.val.empty() || is_option(o.val)) fail("missing value for option '" + o.opt + "'");
    }
    if (it->second.second == OPTIONAL_PARAM && i + 1 < argc &&
        argv[i + 1][0] != '\0' && !is_option(argv[i + 1])) {
      i++;
      o.val = argv[i];
    }
    return o;
  }
  if (is_option(o.str)) {
    size_t pos = o.str.find('=');
    if (pos != std::string::npos) {
      o.opt = o.str.substr(0, pos);
      o.val = o.str.substr(pos + 1);
      if (!m.count(o.opt)) fail("unrecognized option '" + o.opt + "'");
    } else {
      pos = o.str.find_first_of("0123456789");
      if (pos == std::string::npos) o.opt = o.str;
      else { o.opt = o.str.substr(0, pos); o.val = o.str.substr(pos); }
      if (!m.count(o.opt)) fail("unrecognized option '" + o.str + "'");
    }
    if (o.val.empty() && m.at(o.opt).second == REQUIRED_PARAM)
      fail("missing value for option '" + o.opt + "'");
    return o;
  }
  // a number or an integer arithmetic expression
  o.opt = "--number";
  o.val = o.str;
  if (o.str.find_first_of("0123456789") == std::string::npos || o.str[0] == '-')
    fail("unrecognized option '" + o.str + "'");
  return o;
}

uint64_t eval_u64(const Parsed& o) {
  try {
    return psg::calculator::eval_u64(o.val);
  } catch (const std::exception& e) {
    fail("invalid option '" + o.opt + "=" + o.val + "'\n" + e.what());
  }
}

int eval_int(const Parsed& o) {
  const uint64_t v = eval_u64(o);
  if (v > 0x7fffffffull) fail("invalid option '" + o.opt + "=" + o.val + "'\nvalue too large");
  return (int) v;
}

Options parse(int argc, char** argv) {
  Options opts;
  for (int i = 1; i < argc; i++) {
    Parsed o = parse_one(argc, argv, i);
    switch (option_map().at(o.opt).first) {
      case OPT_COUNT: {                                   // CmdOptions.cpp:248-269
        if (o.val.empty()) o.val = "1";
        for (int n = eval_int(o); n > 0; n /= 10) {
          const int d = n % 10;
          if (d < 1 || d > 6) fail("invalid option '" + o.str + "'");
          opts.flags |= 1 << (d - 1);
        }
        break;
      }
      case OPT_DIST: {                                    // CmdOptions.cpp:271-280
        const uint64_t start = opts.numbers.empty() ? 0 : opts.numbers[0];
        opts.numbers.push_back(start + eval_u64(o));
        break;
      }
      case OPT_GPU: opts.gpu = true; break;
      case OPT_GPU_DEVICE: opts.gpu_device = eval_int(o); opts.gpu = true; break;
      case OPT_GPU_INFO: opts.gpu_info = true; break;
      case OPT_HELP: opts.help = true; break;
      case OPT_NUMBER: opts.numbers.push_back(eval_u64(o)); break;
      case OPT_QUIET: opts.quiet = true; break;
      case OPT_SIZE: primesieve::set_sieve_size(eval_int(o)); break;
      case OPT_THREADS: primesieve::set_num_threads(eval_int(o)); break;
      case OPT_TIME: opts.time = true; break;
      case OPT_VERSION: opts.version = true; break;
      case OPT_NO_STATUS: break;
      case OPT_NTH_PRIME: opts.nth_prime = true; break;
      case OPT_PRINT:                                     // CmdOptions.cpp:282-300
        if (!o.val.empty() && eval_int(o) != 1)
          fail("option '" + o.opt + "=" + o.val + "' is not supported: this build prints primes only");
        opts.print = true;
        break;
      case OPT_UNSUPPORTED:
        fail("option '" + o.opt + "' is not supported: this primesieve build counts "
             "primes and prime k-tuplets on the GPU only");
    }
  }
  if (!opts.quiet) opts.time = true;                      // CmdOptions.cpp:395-398
  return opts;
}

void help(int code) {
  std::cout <<
    "Usage: primesieve [START] STOP [OPTION]...\n"
    "Count the primes and/or prime k-tuplets inside [START, STOP]\n"
    "(< 2^64) on an NVIDIA B200 GPU using the segmented sieve of Eratosthenes.\n"
    "\n"
    "Options:\n"
    "  -c, --count[=NUM+]         Count primes and/or prime k-tuplets, NUM <= 6.\n"
    "                             Count primes: -c or --count (default option),\n"
    "                             count twin primes: -c2 or --count=2,\n"
    "                             count prime triplets: -c3 or --count=3, ...\n"
    "                             All requested counts come from one GPU pass.\n"
    "  -d, --dist=DIST            Sieve the interval [START, START + DIST].\n"
    "  -g, --gpu                  Count on the GPU (always the case in this build).\n"
    "      --gpu-device=NUM       Use GPU device NUM, as listed by --gpu-info.\n"
    "      --gpu-info             Print the available GPU devices.\n"
    "  -h, --help                 Print this help menu.\n"
    "  -n, --nth-prime            Find the nth prime, e.g. 100 -n finds the 100th\n"
    "                             prime; with 2 numbers N START finds the nth\n"
    "                             prime > START.\n"
    "  -p, --print                Print the primes inside [START, STOP].\n"
    "  -q, --quiet                Quiet mode, prints less output.\n"
    "  -s, --size=SIZE            Accepted for compatibility (CPU sieve size).\n"
    "  -t, --threads=NUM          Accepted for compatibility (CPU threads).\n"
    "      --time                 Print the time elapsed in seconds.\n"
    "  -v, --version              Print version and license information."
    << std::endl;
  std::exit(code);
}

// primesieve N [START] --nth-prime (reference main.cpp:256-290)
int nth_prime_mode(const Options& opts) {
  if (opts.numbers.empty()) fail("missing n number");
  const int64_t n = (int64_t) opts.numbers[0];
  const uint64_t start = opts.numbers.size() > 1 ? opts.numbers[1] : 0;
  primesieve::set_gpu_device(opts.gpu_device);
  primesieve::set_gpu_enabled(true);
  const std::string dev = primesieve::gpu_active_device();
  if (dev.empty()) fail("could not initialise a GPU: " + primesieve::gpu_last_error());
  if (!opts.quiet) std::cout << "GPU = " << dev << std::endl;
  const auto t0 = std::chrono::steady_clock::now();
  const uint64_t p = primesieve::nth_prime(n, start);
  const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (opts.time)
    std::cout << "Seconds: " << std::fixed << std::setprecision(3) << seconds << std::endl;
  if (opts.quiet) std::cout << p << std::endl;
  else std::cout << "Nth prime: " << p << std::endl;
  return 0;
}

int run(int argc, char** argv) {
  if (argc <= 1) help(1);
  Options opts = parse(argc, argv);
  if (opts.help) help(0);
  if (opts.version) {
    std::cout << "primesieve " << primesieve::primesieve_version()
              << " (B200 GPU counting build)" << std::endl;
    return 0;
  }
  if (opts.gpu_info) {                                    // main.cpp:434-450
    std::vector<std::string> devices = primesieve::gpu_devices();
    if (devices.empty()) {
      std::cout << "No GPU devices found." << std::endl;
      return 0;
    }
    std::cout << "GPU devices:" << std::endl;
    for (const std::string& d : devices) std::cout << d << std::endl;
    return 0;
  }
  if (opts.nth_prime) return nth_prime_mode(opts);
  if (opts.numbers.empty()) fail("missing STOP number");
  uint64_t start = 0, stop = opts.numbers[0];
  if (opts.numbers.size() >= 2) { start = opts.numbers[0]; stop = opts.numbers[1]; }
  if (opts.flags == 0) opts.flags = 1;                    // count primes by default

  primesieve::set_gpu_device(opts.gpu_device);
  primesieve::set_gpu_enabled(true);
  const std::string dev = primesieve::gpu_active_device();
  if (dev.empty()) fail("could not initialise a GPU: " + primesieve::gpu_last_error());
  if (!opts.quiet) std::cout << "GPU = " << dev << std::endl;

  if (opts.print) {                                       // primes, one per line
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<uint64_t> primes;
    primesieve::generate_primes(start, stop, &primes);
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::string buf;
    for (uint64_t p : primes) { buf += std::to_string(p); buf += '\n'; }
    std::cout << buf;
    if (opts.time)
      std::cout << "Seconds: " << std::fixed << std::setprecision(3) << seconds << std::endl;
    return 0;
  }

  const auto t0 = std::chrono::steady_clock::now();
  const std::array<uint64_t, 6> counts = primesieve::count_all(start, stop);
  const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  static const char* labels[6] = { "Primes: ", "Twin primes: ", "Prime triplets: ",
                                   "Prime quadruplets: ", "Prime quintuplets: ",
                                   "Prime sextuplets: " };
  if (opts.time)
    std::cout << "Seconds: " << std::fixed << std::setprecision(3) << seconds << std::endl;
  int n = 0;
  for (int i = 0; i < 6; i++) n += (opts.flags >> i) & 1;
  for (int i = 0; i < 6; i++) {
    if (!((opts.flags >> i) & 1)) continue;
    if (opts.quiet && n == 1) std::cout << counts[i] << std::endl;
    else std::cout << labels[i] << counts[i] << std::endl;
  }
  return 0;
}

} // namespace

int main(int argc, char** argv) {
  try {
    return run(argc, argv);
  } catch (const std::exception& e) {
    std::cerr << "primesieve: " << e.what() << std::endl
              << "Try 'primesieve --help' for more information." << std::endl;
    return 1;
  }
}
