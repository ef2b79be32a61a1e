// Minimal stand-in for the Tiny Shading Language argument header.
// Only the value types that SORT's math/spectrum headers convert from are
// declared here; no shader can be compiled or run through this stub.
// Test infrastructure for the oracle build; never part of the product.
#pragma once
#include <memory>
#include <string>

namespace Tsl_Namespace {
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
}
using Tsl_float3 = Tsl_Namespace::float3;
using Tsl_float  = float;
using Tsl_int    = int;
using Tsl_bool   = bool;
using Tsl_double = double;
using Tsl_resource = void*;
