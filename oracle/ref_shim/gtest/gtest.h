/* Minimal stand-in for <gtest/gtest.h> so that reference test files compile
 * as plain translation units; TEST bodies become uncalled functions and only
 * the CPU twins defined beside them are used (oracle/ref_build.sh). */
#ifndef ORACLE_SHIM_GTEST_H
#define ORACLE_SHIM_GTEST_H
#define TEST(suite, name) void shim_test_##suite##_##name()
#define ASSERT_TRUE(x) (void)(x)
#define ASSERT_FALSE(x) (void)(x)
namespace testing {
struct Environment {
    virtual void SetUp() {}
    virtual void TearDown() {}
    virtual ~Environment() {}
};
inline void InitGoogleTest(int *, char **) {}
inline Environment *AddGlobalTestEnvironment(Environment *e) { return e; }
}  // namespace testing
#define RUN_ALL_TESTS() 0
#endif
