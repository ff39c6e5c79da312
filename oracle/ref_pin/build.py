"""TEST INFRASTRUCTURE: build the reference's own hot-path kernels into oracle/_ref/libsv_refpin.so.

This is the recipe that pins the oracle to the reference. The reference (oojimaflib/mfcm) is a
hipSYCL project whose build needs AdaptiveCpp, Boost and a clang front end, none of which is
in this image; its kernel functors, however, are plain C++ templates over SYCL accessors. The
recipe:

  1. copies the reference source files that define the hot path, unchanged apart from the two
     mechanical patches below, from the reference tree into oracle/_ref/src/ (same layout;
     oracle/_ref/ is git-ignored, so no reference source enters the repository);
  2. puts stand-ins from oracle/ref_pin/stubs/ at the places of the headers that the hot path
     includes but does not use (configuration, geometry, field generators, output files);
  3. compiles oracle/ref_pin/ref_pin.cpp -- this project's driver, which creates meshes,
     fields and states through the reference's own classes and launches the reference's own
     kernel functors through a host-only SYCL stand-in (oracle/ref_pin/shim/CL/sycl.hpp) --
     with the same flags as the oracle (-O2 -ffp-contract=off: separately rounded IEEE
     operations, as the reference's CPU arithmetic).

Patches, both forced by g++ (which does not accept explicit specialisations at class scope,
a clang extension the reference relies on):
  * src/Mesh/Cartesian2DMesh.hpp: each member-template specialisation written inside the two
    mesh classes is moved, unchanged, to namespace scope after its class (qualified with the
    class name); the geometry include, which the mesh never uses, is dropped;
  * src/SaintVenant/{State,Fluxes}.hpp: the in-class specialisation of the output-field lookup
    (get_output_field_ptr) is folded into its primary template as an `if constexpr` branch
    (same lookup); src/SaintVenant/SourceTerm.hpp: its three lookup specialisations, which
    only name fields for output files, are removed.

Everything else is compiled as the reference wrote it. Without the reference tree (the GPU
machines do not have it) `available()` is False and the pin tests skip.

A second library, oracle/_ref/libsv_refpin_nimrod.so, holds the reference's NIMROD raster reader
(src/Raster/RasterFormats/NIMROD.cpp with src/Raster/RasterFormat.hpp, copied unchanged) and
oracle/ref_pin/nimrod_pin.cpp, the driver that runs it on a file and copies out what it read.
A third, oracle/_ref/libsv_refpin_ts.so, holds the reference's time-series reader
(src/Input/TimeSeries.cpp and .hpp with the rapidcsv header the reference vendors, copied
unchanged into a tree of their own) and oracle/ref_pin/ts_pin.cpp, its driver.
"""
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_SRC = os.environ.get("MFCM_REFERENCE_SRC", "/root/reference/src")
OUT = os.path.join(REPO, "oracle", "_ref")
TREE = os.path.join(OUT, "src")
LIB = os.path.join(OUT, "libsv_refpin.so")

# reference files compiled into the pin, relative to the reference's src/
COPY = [
    "sycl.hpp",
    "DataArray/DataArray.hpp", "DataArray/DataArray.cpp",
    "Mesh/Mesh.hpp", "Mesh/Cartesian2DMesh.hpp", "Mesh/Cartesian2DMesh.cpp", "Mesh/MeshSelection.hpp",
    "Field/Field.hpp", "Field/Field.cpp", "Field/FieldOperators.hpp", "Field/FieldOperators.cpp",
    "Field/BinaryFieldOperator_impl.hpp",
    "SpatialDerivative/Minmod3.hpp", "SpatialDerivative/SpatialDerivative.hpp",
    "SpatialDerivative/SpatialDerivative.cpp",
    "SaintVenant/State.hpp", "SaintVenant/State.cpp", "SaintVenant/Constants.hpp",
    "SaintVenant/Fluxes.hpp", "SaintVenant/Fluxes.cpp",
    "SaintVenant/FluxKernel.hpp", "SaintVenant/FluxKernel.cpp",
    "SaintVenant/TemporalDerivativeKernel.hpp", "SaintVenant/TemporalDerivativeKernel.cpp",
    "SaintVenant/SourceTerm.hpp",
    "SaintVenant/SourceTerms/ManningRoughnessSourceTerm.hpp",
    "SaintVenant/SourceTerms/ManningRoughnessSourceTerm.cpp",
    "SaintVenant/Boundaries/BoundarySourceTerm.hpp",
    "SaintVenant/Boundaries/DischargeBoundarySourceTerm.hpp",
    "SaintVenant/Boundaries/DischargeBoundarySourceTerm.cpp",
    "SaintVenant/Boundaries/HeadBoundarySourceTerm.hpp",
    "SaintVenant/Boundaries/HeadBoundarySourceTerm.cpp",
    "SaintVenant/SourceTerms/EnergyLossSourceTerm.hpp", "SaintVenant/SourceTerms/EnergyLossSourceTerm.cpp",
    "SaintVenant/SourceTerms/InfiltrationSourceTerm.hpp", "SaintVenant/SourceTerms/InfiltrationSourceTerm.cpp",
    "SaintVenant/SourceTerms/EddyViscositySourceTerm.hpp", "SaintVenant/SourceTerms/EddyViscositySourceTerm.cpp",
    "SaintVenant/Boundaries/StageBoundarySourceTerm.hpp", "SaintVenant/Boundaries/StageBoundarySourceTerm.cpp",
    "Output/OutputFunction.hpp", "Output/OutputFormat.hpp",
    "Config/TimeParameters.hpp", "Config/TimeParameters.cpp",
    "TemporalScheme/TemporalScheme.hpp", "TemporalScheme/RungeKutta.hpp", "TemporalScheme/RungeKutta.cpp",
]
# the NIMROD reader, compiled into its own library
NIMROD_COPY = ["Raster/RasterFormat.hpp", "Raster/RasterFormats/NIMROD.hpp", "Raster/RasterFormats/NIMROD.cpp"]
# the time-series reader, compiled into its own library from a tree of its own (the kernels'
# tree has a stand-in at Input/TimeSeries.hpp): destination -> reference source file
TS_COPY = {"tsreal/Input/TimeSeries.hpp": "Input/TimeSeries.hpp", "tsreal/Input/TimeSeries.cpp": "Input/TimeSeries.cpp",
           "tsreal/rapidcsv/rapidcsv.h": "rapidcsv/rapidcsv.h"}
# stand-ins, by the path the reference includes them from
STUBS = {
    "Config/Config.hpp": "Config.hpp",
    "Config/TimeParser.hpp": "TimeParser.hpp",
    "Geometry/Geometry.hpp": "Geometry.hpp",
    "Input/FieldGenerator.hpp": "FieldGenerator.hpp",
    "Input/TimeSeries.hpp": "TimeSeries.hpp",
    "Output/CheckFile.hpp": "CheckFile.hpp",
    "Output/OutputFile.hpp": "OutputFile.hpp",
}
INCLUDE_DIRS = ["", "DataArray", "Mesh", "Field", "SpatialDerivative", "SaintVenant", "SaintVenant/SourceTerms",
                "SaintVenant/Boundaries", "Config", "Geometry", "Input", "Output", "TemporalScheme",
                "Raster", "Raster/RasterFormats"]
FLAGS = ["-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-w"]
DRIVER = os.path.join(HERE, "ref_pin.cpp")
NIMROD_DRIVER = os.path.join(HERE, "nimrod_pin.cpp")
NIMROD_LIB = os.path.join(OUT, "libsv_refpin_nimrod.so")
TS_DRIVER = os.path.join(HERE, "ts_pin.cpp")
TS_LIB = os.path.join(OUT, "libsv_refpin_ts.so")


def available():
    return os.path.isdir(REF_SRC) and all(os.path.exists(os.path.join(REF_SRC, f))
                                          for f in COPY + NIMROD_COPY + list(TS_COPY.values()))


def _block_end(text, start):
    """Index just past the brace-balanced body that starts at the first '{' after `start`."""
    i = text.index("{", start)
    depth = 0
    while True:
        c = text[i]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return i + 1
        i += 1


def _class_span(text, name):
    """(start of body, index of the closing brace) of `class name {...};`."""
    m = re.search(r"\bclass\s+%s\s*\n?\s*\{" % re.escape(name), text)
    if not m:
        raise RuntimeError(f"class {name} not found")
    end = _block_end(text, m.start())
    return m.end(), end - 1


def move_specialisations_out(text, cls):
    """Move every `template<> ... { ... }` inside class `cls` to namespace scope after it."""
    body_start, body_end = _class_span(text, cls)
    body = text[body_start:body_end]
    moved = []
    out = []
    pos = 0
    for m in re.finditer(r"template\s*<\s*>", body):
        if m.start() < pos:
            continue
        end = _block_end(body, m.end())
        spec = body[m.end():end]
        # RET NAME<ARGS>(PARAMS) const { BODY }  ->  RET cls::NAME<ARGS>(PARAMS) const { BODY }
        fm = re.search(r"(\w+)\s*<\s*MeshComponent::", spec)
        if not fm:
            raise RuntimeError(f"unexpected specialisation in {cls}: {spec[:80]!r}")
        ret = spec[:fm.start()]
        ret = re.sub(r"\boffset_type\b", f"{cls}::offset_type", ret)
        moved.append("template<>" + ret + f"{cls}::" + spec[fm.start():])
        out.append(body[pos:m.start()])
        pos = end
    out.append(body[pos:])
    close = text.index(";", body_end) + 1
    return text[:body_start] + "".join(out) + text[body_end:close] + "\n\n" + "\n\n".join(moved) + "\n" + text[close:]


def drop_specialisations(text):
    """Remove every `template<> ... { ... }` (in-class output-field lookups)."""
    while True:
        m = re.search(r"template\s*<\s*>", text)
        if not m:
            return text
        text = text[:m.start()] + text[_block_end(text, m.end()):]


def merge_lookup_specialisation(text):
    """Fold the one in-class specialisation `template<> F* get_output_field_ptr<F>(...) {B}` into
    its primary template `template<typename O> O* get_output_field_ptr(...) { return nullptr; }`
    as `if constexpr (std::is_same<O, F>::value) {B} else { return nullptr; }`: the same lookup,
    in a form g++ accepts."""
    m = re.search(r"template\s*<\s*>\s*(\w+)\s*\*\s*get_output_field_ptr\s*<\s*(\w+)\s*>\s*\([^)]*\)\s*", text)
    if not m:
        raise RuntimeError("output-field lookup specialisation not found")
    end = _block_end(text, m.end())
    body = text[text.index("{", m.end()):end]
    arg = m.group(2)
    text = text[:m.start()] + text[end:]
    pm = re.search(r"template\s*<\s*typename\s+(\w+)\s*>\s*\1\s*\*\s*get_output_field_ptr\s*\([^)]*\)\s*", text)
    if not pm:
        raise RuntimeError("output-field lookup template not found")
    pend = _block_end(text, pm.end())
    merged = "{\n    if constexpr (std::is_same<%s, %s>::value) %s else { return nullptr; }\n  }" % (pm.group(1), arg, body)
    return text[:text.index("{", pm.end())] + merged + text[pend:]


def patch(rel, text):
    if rel == "Mesh/Cartesian2DMesh.hpp":
        text = text.replace('#include "../Geometry/Geometry.hpp"', "")
        text = move_specialisations_out(text, "Cartesian2DMesh")
        text = move_specialisations_out(text, "Cartesian2DMeshAccessor")
    elif rel in ("SaintVenant/State.hpp", "SaintVenant/Fluxes.hpp"):
        text = "#include <type_traits>\n" + merge_lookup_specialisation(text)
    elif rel == "SaintVenant/SourceTerm.hpp":
        text = drop_specialisations(text)
    return text


def prepare():
    if os.path.isdir(TREE):
        shutil.rmtree(TREE)
    for rel in COPY + NIMROD_COPY:
        dst = os.path.join(TREE, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        with open(os.path.join(REF_SRC, rel)) as f:
            text = f.read()
        with open(dst, "w") as f:
            f.write(patch(rel, text))
    for rel, stub in STUBS.items():
        dst = os.path.join(TREE, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        shutil.copy(os.path.join(HERE, "stubs", stub), dst)
    # the time-series tree: the reference's reader and rapidcsv unchanged, the check-file stand-in
    for dst_rel, src_rel in TS_COPY.items():
        dst = os.path.join(TREE, dst_rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        shutil.copy(os.path.join(REF_SRC, src_rel), dst)
    dst = os.path.join(TREE, "tsreal", "Output", "CheckFile.hpp")
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    shutil.copy(os.path.join(HERE, "stubs", "CheckFile.hpp"), dst)


def _stale(lib, driver, copied):
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [driver, os.path.join(HERE, "shim", "CL", "sycl.hpp"), __file__]
    deps += [os.path.join(HERE, "stubs", s) for s in STUBS.values()]
    deps += [os.path.join(REF_SRC, f) for f in copied]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Build both pin libraries (when stale); returns the path of the kernels' library."""
    if not available():
        raise RuntimeError(f"reference sources not found under {REF_SRC}")
    targets = [(LIB, DRIVER, COPY), (NIMROD_LIB, NIMROD_DRIVER, COPY + NIMROD_COPY),
               (TS_LIB, TS_DRIVER, COPY + list(TS_COPY.values()))]
    todo = [t for t in targets if force or _stale(*t)]
    if not todo:
        return LIB
    os.makedirs(OUT, exist_ok=True)
    prepare()
    inc = ["-I", os.path.join(HERE, "shim")]
    for d in INCLUDE_DIRS:
        inc += ["-I", os.path.join(TREE, d)]
    for lib, driver, _ in todo:
        first = ["-I", os.path.join(TREE, "tsreal", "Input")] if lib == TS_LIB else []
        cmd = ["g++"] + FLAGS + inc[:2] + first + inc[2:] + [driver, "-o", lib]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


def build_ts(force=False, verbose=False):
    """Build (when stale) and return the path of the time-series reader's library."""
    build(force=force, verbose=verbose)
    return TS_LIB


def build_nimrod(force=False, verbose=False):
    """Build (when stale) and return the path of the NIMROD reader's library."""
    build(force=force, verbose=verbose)
    return NIMROD_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
