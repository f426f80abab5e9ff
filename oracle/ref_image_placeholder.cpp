// Test infrastructure for the oracle build only.
//
// The reference's Mesh (src/painter/shapes/mesh.cpp:104-108,191) references the texture image
// class Image<N> (src/painter/image/image.h:28-68), whose definitions live in
// src/painter/image/image.cpp next to PNG file I/O that needs SFML (not installed here).  Meshes
// built by the oracle never carry images or materials (create_obj_for_facets gives facets with
// material -1, src/obj/create/facets.cpp:203-205), so these members are never called; they are
// defined here only so that the reference objects link, and they fail loudly if ever reached.

#include "painter/image/image.h"

#include "com/error.h"

template <size_t N>
Image<N>::Image(const std::array<int, N>&)
{
        error("oracle build: images are not supported");
}

template <size_t N>
Image<N>::Image(const std::array<int, N>&, const std::vector<unsigned char>&)
{
        error("oracle build: images are not supported");
}

template <size_t N>
template <typename T>
Color Image<N>::texture(const Vector<N, T>&) const
{
        error("oracle build: textures are not supported");
}

template Image<2>::Image(const std::array<int, 2>&, const std::vector<unsigned char>&);
template Image<3>::Image(const std::array<int, 3>&, const std::vector<unsigned char>&);
template Image<4>::Image(const std::array<int, 4>&, const std::vector<unsigned char>&);
template Image<5>::Image(const std::array<int, 5>&, const std::vector<unsigned char>&);

template Color Image<2>::texture(const Vector<2, float>&) const;
template Color Image<3>::texture(const Vector<3, float>&) const;
template Color Image<4>::texture(const Vector<4, float>&) const;
template Color Image<5>::texture(const Vector<5, float>&) const;
template Color Image<2>::texture(const Vector<2, double>&) const;
template Color Image<3>::texture(const Vector<3, double>&) const;
template Color Image<4>::texture(const Vector<4, double>&) const;
template Color Image<5>::texture(const Vector<5, double>&) const;
