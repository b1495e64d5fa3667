# CMake package configuration for the B200 build of AXHEL.
#
#   find_package(AXHEL CONFIG REQUIRED)          # with -DAXHEL_DIR=<repo>/cmake
#   target_link_libraries(seal PUBLIC AXHEL::axhel)
#
# Provides the imported target AXHEL::axhel (the same name the reference
# exports, axhel/CMakeLists.txt) for the shared library axhel_b200/libaxhel.so
# built by `python -m axhel_b200.build`, with the drop-in headers
# (include/axhel/*.hpp, namespace unipi::axhel) and the C-ABI
# (include/axhel_cuda.h).  The library embeds the CUDA runtime; the consumer
# needs a CUDA driver at run time only.
get_filename_component(_AXHEL_ROOT "${CMAKE_CURRENT_LIST_DIR}/.." ABSOLUTE)
set(_AXHEL_LIB "${_AXHEL_ROOT}/axhel_b200/libaxhel.so")
if(NOT EXISTS "${_AXHEL_LIB}")
    set(AXHEL_FOUND FALSE)
    set(AXHEL_NOT_FOUND_MESSAGE "libaxhel.so not built: run python -m axhel_b200.build in ${_AXHEL_ROOT}")
    return()
endif()
if(NOT TARGET AXHEL::axhel)
    add_library(AXHEL::axhel SHARED IMPORTED)
    set_target_properties(AXHEL::axhel PROPERTIES
        IMPORTED_LOCATION "${_AXHEL_LIB}"
        INTERFACE_INCLUDE_DIRECTORIES "${_AXHEL_ROOT}/include"
        INTERFACE_COMPILE_FEATURES cxx_std_17)
endif()
set(AXHEL_VERSION 1.0.0)
set(AXHEL_FOUND TRUE)
