// FieldGenerator.hpp -- TEST INFRASTRUCTURE: stand-in for the reference's configured field
// generators; the pin driver builds fields from arrays instead.
#pragma once
#include "Field.hpp"
template <typename T, typename Mesh, MeshComponent C>
class FieldGenerator;
