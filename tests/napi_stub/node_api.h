// Declarations of the public N-API functions and types that host/napi/addon.cc
// uses (names and signatures as Node publishes them in js_native_api.h and
// node_api.h), so the addon can be syntax-checked where no Node headers exist.
// Test infrastructure only: a real build uses node-gyp and Node's own headers.
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>
typedef struct napi_env__* napi_env;
typedef struct napi_value__* napi_value;
typedef struct napi_callback_info__* napi_callback_info;
typedef enum { napi_ok, napi_invalid_arg } napi_status;
typedef enum { napi_undefined, napi_null, napi_boolean, napi_number, napi_string, napi_symbol, napi_object, napi_function, napi_external, napi_bigint } napi_valuetype;
typedef enum { napi_int8_array, napi_uint8_array, napi_uint8_clamped_array, napi_int16_array, napi_uint16_array, napi_int32_array, napi_uint32_array, napi_float32_array, napi_float64_array, napi_bigint64_array, napi_biguint64_array } napi_typedarray_type;
typedef napi_value (*napi_callback)(napi_env env, napi_callback_info info);
typedef void (*napi_finalize)(napi_env env, void* finalize_data, void* finalize_hint);
typedef enum { napi_default = 0 } napi_property_attributes;
typedef struct { const char* utf8name; napi_value name; napi_callback method; napi_callback getter; napi_callback setter; napi_value value; napi_property_attributes attributes; void* data; } napi_property_descriptor;
extern "C" {
napi_status napi_get_cb_info(napi_env, napi_callback_info, size_t*, napi_value*, napi_value*, void**);
napi_status napi_get_value_external(napi_env, napi_value, void**);
napi_status napi_create_external(napi_env, void*, napi_finalize, void*, napi_value*);
napi_status napi_get_value_double(napi_env, napi_value, double*);
napi_status napi_get_value_int32(napi_env, napi_value, int32_t*);
napi_status napi_get_value_bool(napi_env, napi_value, bool*);
napi_status napi_get_value_string_utf8(napi_env, napi_value, char*, size_t, size_t*);
napi_status napi_has_named_property(napi_env, napi_value, const char*, bool*);
napi_status napi_get_named_property(napi_env, napi_value, const char*, napi_value*);
napi_status napi_set_named_property(napi_env, napi_value, const char*, napi_value);
napi_status napi_is_typedarray(napi_env, napi_value, bool*);
napi_status napi_get_typedarray_info(napi_env, napi_value, napi_typedarray_type*, size_t*, void**, napi_value*, size_t*);
napi_status napi_get_element(napi_env, napi_value, uint32_t, napi_value*);
napi_status napi_typeof(napi_env, napi_value, napi_valuetype*);
napi_status napi_throw_error(napi_env, const char*, const char*);
napi_status napi_throw_type_error(napi_env, const char*, const char*);
napi_status napi_throw_range_error(napi_env, const char*, const char*);
napi_status napi_is_exception_pending(napi_env, bool*);
napi_status napi_create_object(napi_env, napi_value*);
napi_status napi_create_double(napi_env, double, napi_value*);
napi_status napi_get_boolean(napi_env, bool, napi_value*);
napi_status napi_get_null(napi_env, napi_value*);
napi_status napi_define_properties(napi_env, napi_value, size_t, const napi_property_descriptor*);
}
#define NAPI_MODULE_INIT() extern "C" napi_value napi_register_module_v1(napi_env env, napi_value exports)
