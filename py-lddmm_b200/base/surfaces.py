"""Minimal drop-in `Surface` container (reference: base/surfaces.py:226-351, :1645-1655).

Holds what the point-set hot path reads: vertices, faces, vertex weights, face weights, face centres and
surfels (cross(v2-v1, v3-v1)/2). Mesh I/O, remeshing and plotting of the reference are outside this package;
`read_obj` / `read_vtk_ascii` cover plain triangle files.
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
    return np.array(f, dtype=np.int64), np.array(v, dtype=np.float64)


def read_vtk_ascii(path):
    with open(path) as fh:
        tok = fh.read().split()
    i = tok.index('POINTS')
    npts = int(tok[i + 1])
    v = np.array(tok[i + 3:i + 3 + 3 * npts], dtype=np.float64).reshape(npts, 3)
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
