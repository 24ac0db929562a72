// gtest.h -- a minimal test harness with the GoogleTest macro interface, so
// the reference project's own C++ test files (written for GoogleTest, which
// is not installed here) compile unchanged against this repository's
// headers.  Test infrastructure only; written for this repository.
//
// Provided: ::testing::Test (SetUp / TearDown), ::testing::Types, TEST,
// TEST_F, TYPED_TEST_SUITE, TYPED_TEST, GTEST_SKIP, SCOPED_TRACE, and the
// EXPECT_ / ASSERT_ forms of EQ, NE, LT, LE, GT, GE, TRUE, FALSE, NEAR,
// THROW and NO_THROW, each accepting a streamed message.  EXPECT records a
// failure and continues; ASSERT records it and returns from the function;
// GTEST_SKIP marks the test skipped and returns.  main() is in
// gtest_main.cpp: it runs every registered test (or those matching
// --gtest_filter=glob[:glob...]) and exits non-zero if any failed.
#pragma once

#include <cmath>
#include <cstdio>
#include <exception>
#include <functional>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <type_traits>
#include <typeinfo>
#include <utility>
#include <vector>

namespace testing {

class Test {
  public:
    virtual ~Test() = default;
    virtual void SetUp() {}
    virtual void TearDown() {}
    virtual void TestBody() = 0;
};

template <class... Ts>
struct Types {};

namespace internal {

struct TestCase {
    std::string suite, name;
    std::function<std::unique_ptr<Test>()> make;
};

inline std::vector<TestCase> &registry() {
    static std::vector<TestCase> tests;
    return tests;
}

// Outcome of the test that is running.
struct Outcome {
    bool failed = false;
    bool fatal = false;
    bool skipped = false;
    std::vector<std::string> traces;
};
inline Outcome &outcome() {
    static Outcome o;
    return o;
}

struct Message {
    std::ostringstream text;
    template <class X>
    Message &operator<<(const X &x) {
        text << x;
        return *this;
    }
};

// `Failure(...) = Message() << ...` records a failure with the message.
class Failure {
  public:
    Failure(bool fatal, const char *file, int line, std::string what)
        : fatal_(fatal), file_(file), line_(line), what_(std::move(what)) {}
    void operator=(const Message &m) const {
        auto &o = outcome();
        o.failed = true;
        o.fatal = o.fatal || fatal_;
        std::ostringstream out;
        out << file_ << ":" << line_ << ": Failure\n" << what_;
        const std::string extra = m.text.str();
        if (!extra.empty()) out << "\n" << extra;
        for (auto it = o.traces.rbegin(); it != o.traces.rend(); ++it) out << "\n  trace: " << *it;
        std::cout << out.str() << std::endl;
    }

  private:
    bool fatal_;
    const char *file_;
    int line_;
    std::string what_;
};

class Skip {
  public:
    Skip(const char *file, int line) : file_(file), line_(line) {}
    void operator=(const Message &m) const {
        outcome().skipped = true;
        std::cout << file_ << ":" << line_ << ": Skipped " << m.text.str() << std::endl;
    }

  private:
    const char *file_;
    int line_;
};

class ScopedTrace {
  public:
    template <class X>
    ScopedTrace(const char *file, int line, const X &message) {
        std::ostringstream s;
        s << file << ":" << line << ": " << message;
        outcome().traces.push_back(s.str());
    }
    ~ScopedTrace() { outcome().traces.pop_back(); }
    ScopedTrace(const ScopedTrace &) = delete;
    ScopedTrace &operator=(const ScopedTrace &) = delete;
};

template <class X>
std::string show(const X &x) {
    std::ostringstream s;
    if constexpr (requires(std::ostream &os) { os << x; }) {
        if constexpr (std::is_same_v<X, bool>) s << (x ? "true" : "false");
        else s << x;
    } else if constexpr (std::is_enum_v<X>) {
        s << static_cast<long long>(x);
    } else if constexpr (requires { x.begin(); x.end(); }) {
        s << "{";
        bool first = true;
        for (const auto &e : x) {
            s << (first ? "" : ", ") << show(e);
            first = false;
        }
        s << "}";
    } else {
        s << "<" << sizeof(X) << "-byte object>";
    }
    return s.str();
}

struct Check {
    bool ok;
    std::string what;
};

template <class A, class B, class Op>
Check compare(const char *op, const char *ea, const char *eb, const A &a, const B &b, Op pass) {
    if (pass(a, b)) return {true, {}};
    return {false, std::string("Expected: (") + ea + ") " + op + " (" + eb + "), actual: " + show(a) + " vs " + show(b)};
}

inline Check truth(bool value, bool want, const char *expr) {
    if (value == want) return {true, {}};
    return {false, std::string("Value of: ") + expr + "\n  Actual: " + (value ? "true" : "false") +
                       "\nExpected: " + (want ? "true" : "false")};
}

inline Check near(double a, double b, double tol, const char *ea, const char *eb, const char *et) {
    const double diff = std::fabs(a - b);
    if (diff <= tol) return {true, {}};
    std::ostringstream s;
    s.precision(17);
    s << "The difference between " << ea << " and " << eb << " is " << diff << ", which exceeds " << et
      << ", where\n" << ea << " evaluates to " << a << ",\n" << eb << " evaluates to " << b << ", and\n"
      << et << " evaluates to " << tol << ".";
    return {false, s.str()};
}

template <class E, class F>
Check throws(F &&statement, const char *text, const char *type) {
    try {
        statement();
    } catch (const E &) {
        return {true, {}};
    } catch (const std::exception &e) {
        return {false, std::string("Expected: ") + text + " throws an exception of type " + type +
                           ".\n  Actual: it throws a different type: " + e.what()};
    } catch (...) {
        return {false, std::string("Expected: ") + text + " throws an exception of type " + type +
                           ".\n  Actual: it throws a different type."};
    }
    return {false, std::string("Expected: ") + text + " throws an exception of type " + type +
                       ".\n  Actual: it throws nothing."};
}

template <class F>
Check nothrow(F &&statement, const char *text) {
    try {
        statement();
    } catch (const std::exception &e) {
        return {false, std::string("Expected: ") + text + " doesn't throw an exception.\n  Actual: it throws " +
                           e.what()};
    } catch (...) {
        return {false, std::string("Expected: ") + text + " doesn't throw an exception.\n  Actual: it throws."};
    }
    return {true, {}};
}

template <class TestClass>
bool add(const char *suite, const char *name) {
    registry().push_back({suite, name, [] { return std::unique_ptr<Test>(new TestClass); }});
    return true;
}

template <template <class> class TestClass, class... Ts>
bool addTyped(Types<Ts...>, const char *suite, const char *name) {
    int k = 0;
    ((registry().push_back({std::string(suite) + "/" + std::to_string(k++), name,
                            [] { return std::unique_ptr<Test>(new TestClass<Ts>); }})),
     ...);
    return true;
}

}  // namespace internal
}  // namespace testing

#define TF_GTEST_CAT2(a, b) a##b
#define TF_GTEST_CAT(a, b) TF_GTEST_CAT2(a, b)

#define TF_GTEST_CHECK(check, fatal)                                                     \
    if (const ::testing::internal::Check tf_gtest_check = (check); tf_gtest_check.ok) \
        ;                                                                                \
    else                                                                                 \
        TF_GTEST_ON_FAIL_##fatal ::testing::internal::Failure(fatal, __FILE__, __LINE__, tf_gtest_check.what) = \
            ::testing::internal::Message()
#define TF_GTEST_ON_FAIL_true return
#define TF_GTEST_ON_FAIL_false

#define TF_GTEST_CMP(op, a, b, fatal)                                                                            \
    TF_GTEST_CHECK(::testing::internal::compare(#op, #a, #b, (a), (b),                                           \
                                                [](const auto &x, const auto &y) { return x op y; }),             \
                   fatal)

#define EXPECT_EQ(a, b) TF_GTEST_CMP(==, a, b, false)
#define EXPECT_NE(a, b) TF_GTEST_CMP(!=, a, b, false)
#define EXPECT_LT(a, b) TF_GTEST_CMP(<, a, b, false)
#define EXPECT_LE(a, b) TF_GTEST_CMP(<=, a, b, false)
#define EXPECT_GT(a, b) TF_GTEST_CMP(>, a, b, false)
#define EXPECT_GE(a, b) TF_GTEST_CMP(>=, a, b, false)
#define ASSERT_EQ(a, b) TF_GTEST_CMP(==, a, b, true)
#define ASSERT_NE(a, b) TF_GTEST_CMP(!=, a, b, true)
#define ASSERT_LT(a, b) TF_GTEST_CMP(<, a, b, true)
#define ASSERT_LE(a, b) TF_GTEST_CMP(<=, a, b, true)
#define ASSERT_GT(a, b) TF_GTEST_CMP(>, a, b, true)
#define ASSERT_GE(a, b) TF_GTEST_CMP(>=, a, b, true)
#define EXPECT_TRUE(c) TF_GTEST_CHECK(::testing::internal::truth(static_cast<bool>(c), true, #c), false)
#define EXPECT_FALSE(c) TF_GTEST_CHECK(::testing::internal::truth(static_cast<bool>(c), false, #c), false)
#define ASSERT_TRUE(c) TF_GTEST_CHECK(::testing::internal::truth(static_cast<bool>(c), true, #c), true)
#define ASSERT_FALSE(c) TF_GTEST_CHECK(::testing::internal::truth(static_cast<bool>(c), false, #c), true)
#define EXPECT_NEAR(a, b, tol) \
    TF_GTEST_CHECK(::testing::internal::near(double(a), double(b), double(tol), #a, #b, #tol), false)
#define ASSERT_NEAR(a, b, tol) \
    TF_GTEST_CHECK(::testing::internal::near(double(a), double(b), double(tol), #a, #b, #tol), true)
#define EXPECT_THROW(statement, type) \
    TF_GTEST_CHECK(::testing::internal::throws<type>([&] { statement; }, #statement, #type), false)
#define ASSERT_THROW(statement, type) \
    TF_GTEST_CHECK(::testing::internal::throws<type>([&] { statement; }, #statement, #type), true)
#define EXPECT_NO_THROW(statement) \
    TF_GTEST_CHECK(::testing::internal::nothrow([&] { statement; }, #statement), false)
#define ASSERT_NO_THROW(statement) \
    TF_GTEST_CHECK(::testing::internal::nothrow([&] { statement; }, #statement), true)

#define GTEST_SKIP() return ::testing::internal::Skip(__FILE__, __LINE__) = ::testing::internal::Message()
#define SCOPED_TRACE(message) \
    ::testing::internal::ScopedTrace TF_GTEST_CAT(tf_gtest_trace_, __LINE__)(__FILE__, __LINE__, (message))

#define TF_GTEST_CLASS(suite, name) suite##_##name##_Test

#define TEST(suite, name)                                                                                        \
    class TF_GTEST_CLASS(suite, name) : public ::testing::Test {                                                 \
      public:                                                                                                    \
        void TestBody() override;                                                                                \
    };                                                                                                           \
    static const bool TF_GTEST_CAT(tf_gtest_registered_, __LINE__) =                                             \
        ::testing::internal::add<TF_GTEST_CLASS(suite, name)>(#suite, #name);                                    \
    void TF_GTEST_CLASS(suite, name)::TestBody()

#define TEST_F(fixture, name)                                                                                    \
    class TF_GTEST_CLASS(fixture, name) : public fixture {                                                       \
      public:                                                                                                    \
        void TestBody() override;                                                                                \
    };                                                                                                           \
    static const bool TF_GTEST_CAT(tf_gtest_registered_, __LINE__) =                                             \
        ::testing::internal::add<TF_GTEST_CLASS(fixture, name)>(#fixture, #name);                                \
    void TF_GTEST_CLASS(fixture, name)::TestBody()

#define TYPED_TEST_SUITE(fixture, types) using tf_gtest_types_##fixture = types

#define TYPED_TEST(fixture, name)                                                                                \
    template <class tf_gtest_type>                                                                               \
    class TF_GTEST_CLASS(fixture, name) : public fixture<tf_gtest_type> {                                        \
      public:                                                                                                    \
        using TypeParam = tf_gtest_type;                                                                         \
        void TestBody() override;                                                                                \
    };                                                                                                           \
    static const bool TF_GTEST_CAT(tf_gtest_registered_, __LINE__) =                                             \
        ::testing::internal::addTyped<TF_GTEST_CLASS(fixture, name)>(tf_gtest_types_##fixture{}, #fixture, #name); \
    template <class tf_gtest_type>                                                                               \
    void TF_GTEST_CLASS(fixture, name)<tf_gtest_type>::TestBody()
