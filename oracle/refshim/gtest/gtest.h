// Minimal GoogleTest-compatible harness used only to run the reference's own
// unit/integration/regression test sources (tests/*/*.cpp of gdeskos/DVMpp)
// against the oracle build.  Test infrastructure, not product code.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace testing {
class Test {
  public:
    virtual ~Test() = default;
    virtual void SetUp() {}
    virtual void TearDown() {}
    virtual void TestBody() = 0;
};
struct Registered {
    std::string name;
    std::function<Test*()> make;
};
inline std::vector<Registered>& registry() {
    static std::vector<Registered> r;
    return r;
}
inline int& failures() {
    static int f = 0;
    return f;
}
struct Registrar {
    Registrar(const char* suite, const char* name, std::function<Test*()> make) {
        registry().push_back({std::string(suite) + "." + name, make});
    }
};
inline void report(const char* file, int line, const std::string& what) {
    ++failures();
    std::cerr << file << ":" << line << ": Failure: " << what << "\n";
}
inline bool almost_equal_ulps(double a, double b) {
    if (a == b) return true;
    if (std::isnan(a) || std::isnan(b)) return false;
    long long ia, ib;
    static_assert(sizeof(double) == sizeof(long long), "size");
    std::memcpy(&ia, &a, 8);
    std::memcpy(&ib, &b, 8);
    if ((ia < 0) != (ib < 0)) return false;
    long long d = ia > ib ? ia - ib : ib - ia;
    return d <= 4;
}
inline int RunAllTests() {
    int failed_tests = 0;
    for (auto& r : registry()) {
        const int before = failures();
        std::cout << "[ RUN      ] " << r.name << std::endl;
        Test* t = r.make();
        try {
            t->SetUp();
            t->TestBody();
            t->TearDown();
        } catch (const std::exception& e) {
            report("<test>", 0, std::string("uncaught exception: ") + e.what());
        }
        delete t;
        if (failures() != before) {
            ++failed_tests;
            std::cout << "[  FAILED  ] " << r.name << std::endl;
        } else {
            std::cout << "[       OK ] " << r.name << std::endl;
        }
    }
    std::cout << "[==========] " << registry().size() << " tests, " << failed_tests << " failed"
              << std::endl;
    return failed_tests == 0 ? 0 : 1;
}
inline void InitGoogleTest(int*, char**) {}
}  // namespace testing

#include <cstring>

#define DVM_GT_CLASS(suite, name) suite##_##name##_Test
#define TEST_F(suite, name)                                                          \
    class DVM_GT_CLASS(suite, name) : public suite {                                 \
      public:                                                                        \
        void TestBody() override;                                                    \
    };                                                                               \
    static ::testing::Registrar DVM_GT_CLASS(suite, name##_reg)(                     \
        #suite, #name, [] { return static_cast<::testing::Test*>(new DVM_GT_CLASS(suite, name)); }); \
    void DVM_GT_CLASS(suite, name)::TestBody()
#define TEST(suite, name)                                                            \
    class DVM_GT_CLASS(suite, name) : public ::testing::Test {                       \
      public:                                                                        \
        void TestBody() override;                                                    \
    };                                                                               \
    static ::testing::Registrar DVM_GT_CLASS(suite, name##_reg)(                     \
        #suite, #name, [] { return static_cast<::testing::Test*>(new DVM_GT_CLASS(suite, name)); }); \
    void DVM_GT_CLASS(suite, name)::TestBody()

#define DVM_GT_CHECK(cond, text, fatal)                                              \
    do {                                                                             \
        if (!(cond)) {                                                               \
            ::testing::report(__FILE__, __LINE__, text);                             \
            if (fatal) return;                                                       \
        }                                                                            \
    } while (0)
#define DVM_GT_CMP(a, op, b, fatal) DVM_GT_CHECK(((a)op(b)), #a " " #op " " #b, fatal)
#define EXPECT_EQ(a, b) DVM_GT_CMP(a, ==, b, false)
#define EXPECT_NE(a, b) DVM_GT_CMP(a, !=, b, false)
#define EXPECT_GT(a, b) DVM_GT_CMP(a, >, b, false)
#define EXPECT_LT(a, b) DVM_GT_CMP(a, <, b, false)
#define EXPECT_GE(a, b) DVM_GT_CMP(a, >=, b, false)
#define EXPECT_LE(a, b) DVM_GT_CMP(a, <=, b, false)
#define ASSERT_EQ(a, b) DVM_GT_CMP(a, ==, b, true)
#define ASSERT_NE(a, b) DVM_GT_CMP(a, !=, b, true)
#define ASSERT_GT(a, b) DVM_GT_CMP(a, >, b, true)
#define EXPECT_TRUE(c) DVM_GT_CHECK((c), #c, false)
#define EXPECT_FALSE(c) DVM_GT_CHECK(!(c), "!" #c, false)
#define ASSERT_TRUE(c) DVM_GT_CHECK((c), #c, true)
#define EXPECT_NEAR(a, b, tol) DVM_GT_CHECK(std::abs((double)(a) - (double)(b)) <= (tol), "|" #a " - " #b "| <= " #tol, false)
#define EXPECT_DOUBLE_EQ(a, b) DVM_GT_CHECK(::testing::almost_equal_ulps((a), (b)), #a " ~= " #b, false)
#define SUCCEED() do {} while (0)
#define EXPECT_THROW(stmt, exc)                                                      \
    do {                                                                             \
        bool dvm_caught = false;                                                     \
        try { stmt; } catch (const exc&) { dvm_caught = true; } catch (...) {}       \
        DVM_GT_CHECK(dvm_caught, "expected " #exc, false);                           \
    } while (0)
#define EXPECT_NO_THROW(stmt)                                                        \
    do {                                                                             \
        bool dvm_threw = false;                                                      \
        try { stmt; } catch (...) { dvm_threw = true; }                              \
        DVM_GT_CHECK(!dvm_threw, "unexpected exception", false);                     \
    } while (0)
