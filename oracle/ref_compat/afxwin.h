#pragma once
#include "afx_stubs.h"
