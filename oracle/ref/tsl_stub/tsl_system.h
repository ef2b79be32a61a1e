// Minimal stand-in for the Tiny Shading Language system header.
// Declares the opaque types SORT's material headers name and turns the
// closure/global declaration macros into plain aggregate structs, so that
// SORT's BxDF constructors can be called directly with parameter structs.
// Oracle build only: shaders cannot be compiled or executed with it.
#pragma once
#include "tsl_args.h"
#include <memory>
#include <string>

namespace Tsl_Namespace {
class ShadingContext;
class ShaderInstance;
class ShaderUnitTemplate;
class ShaderGroupTemplate;
struct ClosureTreeNodeBase { int id = 0; };
typedef void* ClosureParamPtr;
typedef int ClosureID;
struct ShaderUnitInputDefaultValue { float x = 0, y = 0, z = 0, w = 0; };
enum TSL_RESOLVING_STATUS { TSL_RESOLVING_SUCCEED = 0 };
class ShadingSystem {
public:
    static ShadingSystem& get_instance() { static ShadingSystem s; return s; }
    std::shared_ptr<ShadingContext> make_shading_context() { return nullptr; }
};
}

#define DECLARE_TSLGLOBAL_BEGIN(T)        struct T {
#define DECLARE_TSLGLOBAL_VAR(type, name)     type name;
#define DECLARE_TSLGLOBAL_END()           };
#define IMPLEMENT_TSLGLOBAL_BEGIN(T)
#define IMPLEMENT_TSLGLOBAL_VAR(type, name)
#define IMPLEMENT_TSLGLOBAL_END()

#define DECLARE_CLOSURE_TYPE_BEGIN(T, name)   struct T {
#define DECLARE_CLOSURE_TYPE_VAR(T, type, v)      type v;
#define DECLARE_CLOSURE_TYPE_END(T)               static int RegisterClosure(); };
#define IMPLEMENT_CLOSURE_TYPE_BEGIN(T)       int T::RegisterClosure() { return 0; }
#define IMPLEMENT_CLOSURE_TYPE_VAR(T, type, v)
#define IMPLEMENT_CLOSURE_TYPE_END(T)
