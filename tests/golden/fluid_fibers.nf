%type_of_analysis
2

%type_of_solver
0

%type_of_rhs
0

%voxel_size
1.0989e-06

%solver_tolerance
1e-04

%number_of_iterations
100000

%image_dimensions
100 100 10

%refinement
2

%number_of_materials
2

%properties_of_materials
0
255

%volume_fraction
47.77 52.23

%data_type
uint8

