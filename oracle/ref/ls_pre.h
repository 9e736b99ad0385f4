/*
 * ls_pre.h - TEST INFRASTRUCTURE ONLY: included ahead of the reference's lightslice.cc so
 * that it compiles unmodified with g++:
 *   - mutable_path.h (reached through mesh_view.h) constructs std::exception from a
 *     string, an MSVC extension; within that header the call becomes std::runtime_error.
 *   - lightslice.cc:1796 binds direction_to_square(...)'s temporary to a non-const
 *     Vec2&; the same mapping is offered as a function returning a reference to a
 *     thread-local copy of its result.
 */
#pragma once
#include <stdexcept>
#include <exception>
#define exception(...) runtime_error(__VA_ARGS__)
#include "mutable_path.h"
#undef exception
#include "concentric_mapping.h"
namespace Renzoku {
inline Vec2 &rzk_direction_to_square_lvalue(const Vec3 &v) {
    thread_local Vec2 r;
    r = direction_to_square(v);
    return r;
}
}
#define direction_to_square rzk_direction_to_square_lvalue
