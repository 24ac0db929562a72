// gtest_main.cpp -- runs the tests registered through tests/cxx/gtest/gtest.h.
//   <binary> [--gtest_filter=glob[:glob...]]
// Prints one line per test ([ RUN ] / [ OK ] / [ SKIPPED ] / [ FAILED ]) and
// a summary; exits 1 when a test failed.  Test infrastructure only.
#include <gtest/gtest.h>

#include <cstring>

namespace {

bool glob(const char *p, const char *s) {
    if (!*p) return !*s;
    if (*p == '*') return glob(p + 1, s) || (*s && glob(p, s + 1));
    return *s && (*p == '?' || *p == *s) && glob(p + 1, s + 1);
}

bool selected(const std::string &full, const std::string &filter) {
    if (filter.empty()) return true;
    std::size_t start = 0;
    while (start <= filter.size()) {
        const std::size_t stop = filter.find(':', start);
        const std::string one = filter.substr(start, stop == std::string::npos ? std::string::npos : stop - start);
        if (glob(one.c_str(), full.c_str())) return true;
        if (stop == std::string::npos) break;
        start = stop + 1;
    }
    return false;
}

}  // namespace

int main(int argc, char **argv) {
    std::string filter;
    for (int k = 1; k < argc; ++k)
        if (std::strncmp(argv[k], "--gtest_filter=", 15) == 0) filter = argv[k] + 15;
    int ran = 0, failed = 0, skipped = 0;
    std::vector<std::string> failures;
    for (const auto &t : testing::internal::registry()) {
        const std::string full = t.suite + "." + t.name;
        if (!selected(full, filter)) continue;
        ++ran;
        auto &o = testing::internal::outcome();
        o = {};
        std::cout << "[ RUN      ] " << full << std::endl;
        try {
            auto test = t.make();
            test->SetUp();
            if (!o.skipped && !o.fatal) test->TestBody();
            test->TearDown();
        } catch (const std::exception &e) {
            o.failed = true;
            std::cout << "uncaught exception: " << e.what() << std::endl;
        } catch (...) {
            o.failed = true;
            std::cout << "uncaught exception of unknown type" << std::endl;
        }
        if (o.failed) {
            ++failed;
            failures.push_back(full);
            std::cout << "[  FAILED  ] " << full << std::endl;
        } else if (o.skipped) {
            ++skipped;
            std::cout << "[  SKIPPED ] " << full << std::endl;
        } else {
            std::cout << "[       OK ] " << full << std::endl;
        }
    }
    std::cout << "[==========] " << ran << " tests ran, " << (ran - failed - skipped) << " passed, " << skipped
              << " skipped, " << failed << " failed." << std::endl;
    for (const auto &f : failures) std::cout << "[  FAILED  ] " << f << std::endl;
    return failed ? 1 : 0;
}
