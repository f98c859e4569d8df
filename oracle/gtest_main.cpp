// Entry point for the reference test sources built against refshim/gtest.
#include <gtest/gtest.h>
int main(int argc, char** argv) {
    ::testing::InitGoogleTest(&argc, argv);
    return ::testing::RunAllTests();
}
