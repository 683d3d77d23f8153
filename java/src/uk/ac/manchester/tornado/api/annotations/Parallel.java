package uk.ac.manchester.tornado.api.annotations;

import java.lang.annotation.ElementType;
import java.lang.annotation.Retention;
import java.lang.annotation.RetentionPolicy;
import java.lang.annotation.Target;

/** Stand-in for TornadoVM's loop annotation: no effect (the loops now run as CUDA kernels). */
@Retention(RetentionPolicy.SOURCE)
@Target({ElementType.LOCAL_VARIABLE, ElementType.PARAMETER})
public @interface Parallel {}
