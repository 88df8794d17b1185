// See ../kernel_operator.h.
#pragma once
