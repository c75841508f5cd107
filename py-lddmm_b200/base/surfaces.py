"""Minimal drop-in `Surface` container (reference: base/surfaces.py:226-351, :364-440, :1645-1655).

Holds what the point-set hot path reads: vertices, faces, vertex weights, face weights, face centres and
surfels (cross(v2-v1, v3-v1)/2), and the vertex areas of the output descriptors. Remeshing and plotting of the
reference are outside this package; `read_obj` / `read_vtk_ascii` read plain triangle files without the vtk
library, which the reference needs for them (base/surfaces.py:1880-1980). Like vtk's readers, which store points in
single precision, they round coordinates declared `float` (and every OBJ coordinate) to float32 before widening
them to float64, so a mesh read here has the vertices the reference would have.
"""
import numpy as np


class Surface:
    def __init__(self, surf=None, weights=None):
        if isinstance(surf, (list, tuple)) and not isinstance(surf[0], (Surface, str)):
            self.vertices = np.array(surf[1], dtype=np.float64, copy=True)
            self.faces = np.int_(np.array(surf[0], copy=True))
            self.component = np.zeros(self.faces.shape[0], dtype=int)
            if weights is None:
                self.weights = np.ones(self.vertices.shape[0], dtype=int)
                self.face_weights = np.ones(self.faces.shape[0], dtype=int)
            else:
                self.updateWeights(weights)
            self.computeCentersAreas()
        elif isinstance(surf, Surface):
            self.vertices = np.copy(surf.vertices)
            self.surfel = np.copy(surf.surfel)
            self.faces = np.copy(surf.faces)
            self.centers = np.copy(surf.centers)
            self.component = np.copy(surf.component)
            if weights is None:
                self.weights = np.copy(surf.weights)
                self.face_weights = np.copy(surf.face_weights)
            else:
                self.updateWeights(weights)
        elif isinstance(surf, str):
            self.read(surf)
        elif surf is None:
            self.vertices = np.empty(0)
            self.centers = np.empty(0)
            self.faces = np.empty(0)
            self.surfel = np.empty(0)
            self.component = np.empty(0)
            self.weights = np.empty(0)
            self.face_weights = np.empty(0)
        else:
            raise TypeError('Surface(surf=(faces, vertices) | Surface | filename)')
        self.edges = None
        self.edgeFaces = None
        self.faceEdges = None

    def read(self, filename):
        if filename.endswith('.obj'):
            f, v = read_obj(filename)
        elif filename.endswith('.vtk'):
            f, v = read_vtk_ascii(filename)
        else:
            raise NameError('Unknown Surface Extension: ' + filename)
        self.__init__(surf=(f, v))

    def computeCentersAreas(self):
        x1, x2, x3 = (self.vertices[self.faces[:, j], :] for j in range(3))
        self.centers = (x1 + x2 + x3) / 3
        self.surfel = np.cross(x2 - x1, x3 - x1) / 2
        w = self.weights
        self.face_weights = (w[self.faces[:, 0]] + w[self.faces[:, 1]] + w[self.faces[:, 2]]) / 3

    def updateWeights(self, w0):
        self.weights = np.copy(w0)
        w = self.weights
        self.face_weights = (w[self.faces[:, 0]] + w[self.faces[:, 1]] + w[self.faces[:, 2]]) / 3

    def updateVertices(self, x0):
        self.vertices = np.array(x0, dtype=np.float64, copy=True)
        x1, x2, x3 = (self.vertices[self.faces[:, j], :] for j in range(3))
        self.centers = (x1 + x2 + x3) / 3
        self.surfel = np.cross(x2 - x1, x3 - x1) / 2

    def surfVolume(self):
        v, f = self.vertices, self.faces
        return float((v[f[:, 0]] * np.cross(v[f[:, 1]], v[f[:, 2]])).sum() / 6)

    def surfArea(self):
        return float(np.sqrt((self.surfel ** 2).sum(axis=1)).sum())

    def saveVTK(self, fileName):
        write_vtk_ascii(fileName, self.faces, self.vertices)

    def computeVertexArea(self, simpleMethod=False):
        """(vertex areas AV, face areas AF) (base/surfaces.py:364-440). simpleMethod: a third of each face's area
        to each corner. Otherwise the mixed rule the reference uses: a face without an obtuse angle gives corner i
        (|e_ij|^2 cot(angle at k) + |e_ik|^2 cot(angle at j)) / 8 (its Voronoi share); a face obtuse at a corner
        gives each other corner |edge to the obtuse corner|^2 / (8 cot(own angle)) and the obtuse corner the rest."""
        V, F = self.vertices, self.faces
        p = [V[F[:, k]] for k in range(3)]
        e12, e13, e23 = p[1] - p[0], p[2] - p[0], p[2] - p[1]
        AF = np.sqrt((np.cross(e12, e13) ** 2).sum(axis=1)) / 2
        AV = np.zeros(V.shape[0])
        if simpleMethod:
            for k in range(3):
                np.add.at(AV, F[:, k], AF / 3)
            return AV, AF
        l12, l13, l23 = (e12 ** 2).sum(1), (e13 ** 2).sum(1), (e23 ** 2).sum(1)
        c1 = (e12 * e13).sum(1) / np.sqrt(l12 * l13)
        c2 = -(e12 * e23).sum(1) / np.sqrt(l12 * l23)
        c3 = (e13 * e23).sum(1) / np.sqrt(l13 * l23)
        cot = [c / np.sqrt(1 - c ** 2) for c in (c1, c2, c3)]
        with np.errstate(divide='ignore', invalid='ignore'):
            u = np.stack([(l12 * cot[2] + l13 * cot[1]) / 8, (l12 * cot[2] + l23 * cot[0]) / 8,
                          (l13 * cot[1] + l23 * cot[0]) / 8], axis=1)
            ob1 = np.stack([AF - l12 / (8 * cot[1]) - l13 / (8 * cot[2]), l12 / (8 * cot[1]), l13 / (8 * cot[2])], 1)
            ob2 = np.stack([l12 / (8 * cot[0]), AF - l12 / (8 * cot[0]) - l23 / (8 * cot[2]), l23 / (8 * cot[2])], 1)
            ob3 = np.stack([l13 / (8 * cot[0]), l23 / (8 * cot[1]), AF - l13 / (8 * cot[0]) - l23 / (8 * cot[1])], 1)
        u = np.where((c1 < 0)[:, None], ob1, np.where((c2 < 0)[:, None], ob2, np.where((c3 < 0)[:, None], ob3, u)))
        for k in range(3):
            np.add.at(AV, F[:, k], u[:, k])
        return AV, AF


def read_obj(path):
    v, f = [], []
    with open(path) as fh:
        for line in fh:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == 'v':
                v.append([float(t) for t in tok[1:4]])
            elif tok[0] == 'f':
                idx = [int(t.split('/')[0]) - 1 for t in tok[1:]]
                for k in range(1, len(idx) - 1):
                    f.append([idx[0], idx[k], idx[k + 1]])
    return np.array(f, dtype=np.int64), np.array(v, dtype=np.float32).astype(np.float64)


def read_vtk_ascii(path):
    with open(path) as fh:
        tok = fh.read().split()
    i = tok.index('POINTS')
    npts = int(tok[i + 1])
    v = np.array(tok[i + 3:i + 3 + 3 * npts], dtype=np.float64).reshape(npts, 3)
    if tok[i + 2].lower() == 'float':
        v = v.astype(np.float32).astype(np.float64)
    j = tok.index('POLYGONS')
    nf = int(tok[j + 1])
    k = j + 3
    faces = []
    for _ in range(nf):
        cnt = int(tok[k])
        idx = [int(t) for t in tok[k + 1:k + 1 + cnt]]
        for q in range(1, cnt - 1):
            faces.append([idx[0], idx[q], idx[q + 1]])
        k += 1 + cnt
    return np.array(faces, dtype=np.int64), v


def write_vtk_ascii(path, faces, vertices):
    with open(path, 'w') as fh:
        fh.write('# vtk DataFile Version 3.0\nsurface\nASCII\nDATASET POLYDATA\n')
        fh.write(f'POINTS {vertices.shape[0]} double\n')
        for p in vertices:
            fh.write(f'{p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n')
        fh.write(f'POLYGONS {faces.shape[0]} {4 * faces.shape[0]}\n')
        for f in faces:
            fh.write(f'3 {f[0]} {f[1]} {f[2]}\n')
