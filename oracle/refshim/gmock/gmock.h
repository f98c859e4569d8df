// Empty stand-in: the reference tests include gmock but use none of it.
#pragma once
#include <gtest/gtest.h>
